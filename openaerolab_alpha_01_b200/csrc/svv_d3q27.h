// svv_d3q27.h — the spectral vanishing viscosity post-pass of D3Q27 levels (host interface).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace oal {

// Enqueue the filter of a stepped level on st: f_out (the step's output) is filtered in place from
// the step's input f_in; n_elements: the element count of each population buffer (index width). storage 0 F32, 1 F16 deviation, 2 BF16 deviation, 3 F64 (OAL_STORE_*);
// nbr: the real topology (-1 = none), indices >= n_real count as none; mslot / cmask: the solid
// masks (bit 13 of a cell's word: the cell is solid). f_post2, when given (same layout as f_out),
// receives the filtered values as well (a caller's f_post_collision). No-op when both strengths
// are 0.
cudaError_t svv_enqueue(int32_t storage, const void* f_in, void* f_out, const PopIndex& pi, int32_t nb,
                        int64_t n_elements, const int32_t* nbr, int32_t n_real, const int32_t* mslot,
                        const uint32_t* cmask, float eps_x, float eps_yz, cudaStream_t st, void* f_post2 = nullptr);

}  // namespace oal
