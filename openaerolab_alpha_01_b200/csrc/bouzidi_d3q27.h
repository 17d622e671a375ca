// bouzidi_d3q27.h — the linear Bouzidi wall correction of D3Q27 levels (host interface).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace oal {

// The boundary cells of one level and their link fractions (device arrays owned by the level).
struct BouzidiSet {
  int32_t n = 0;               // boundary cells
  int2* cells = nullptr;       // (block, cell = x + 8y + 64z), 0-based
  float* q = nullptr;          // [n*27] link fractions (binary16 values widened), direction fastest
  void* vals = nullptr;        // [n*27] corrected populations (compute type) between the two kernels
  float q_min = 0.001f;
  int32_t ff_fallback = 0;     // 0 halfway_bb, 1 wall_eq, 2 bounce_back
  float rel_cap = 0.0f, abs_cap = 0.0f;
};

// Enqueue the correction of the populations f (the step's output, post-collision at every cell)
// on st: storage 0 F32, 1 F16 deviation, 2 BF16 deviation, 3 F64 (OAL_STORE_*). nbr: the real
// topology (-1 = none); indices >= n_real (a pool's ghost blocks) count as none as well.
cudaError_t bouzidi_enqueue(const BouzidiSet& B, int32_t storage, void* f, const PopIndex& pi, const int32_t* nbr,
                            const int32_t* mslot, const uint32_t* cmask, cudaStream_t st, int32_t n_real = 0x7fffffff);

}  // namespace oal
