// pdl.cuh — programmatic dependent launch (sm_90 and later) for chains of small dependent kernels.
//
// A kernel launched with launch_pdl may be scheduled while the previous kernel of its stream (or
// of its CUDA graph) is still running: its CTAs wait in pdl_wait(), its first statement, until that
// kernel has completed and its writes are visible, so the launch latency of the next kernel
// overlaps the tail of the current one. pdl_release() (after the wait) lets the next kernel be
// scheduled early in turn. Kernels launched without the attribute pass both calls at once.
#pragma once

#include <cuda_runtime.h>

#include <utility>

namespace oal {

__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_release() { asm volatile("griddepcontrol.launch_dependents;" :::); }

template <class... KArgs, class... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args&&... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

}  // namespace oal
