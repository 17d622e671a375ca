// noalloc.cu — an FP64 mass/momentum reduction that allocates nothing.
//
// Some callers cannot call cudaMalloc at the point where they need conservation totals: a
// solver step run under a stream-ordered pool that forbids stray allocations, or a host (for
// instance a Julia task holding the GPU through CUDA.jl's allocator) that must not grow device
// memory between steps. `oal_mass_momentum_noalloc` serves them: the
// caller passes the populations and receives {mass, px, py, pz}; the per-block partial sums live
// in a fixed file-scope device array of OAL_NOALLOC_MAX_BLOCKS * 4 doubles (2 MiB) that every GPU
// loading this library holds until the process exits.
//
// The array is shared by all calls on a device and keeps the last call's contents. Every call
// writes each partial it later reads, so nothing has to start at zero; calls that overlap on the
// GPU (two streams at once) race on the array and must be serialised by the caller.
//
// In host code the array's name is only a host-side stand-in, so its device address is fetched
// with cudaGetSymbolAddress once per device, with that device current, by the first call on that
// device. That first call should therefore come before any stream capture.
#include <cuda_runtime.h>
#include <mutex>
#include <cstdarg>
#include <cstdio>
#include <string>

#include "common.cuh"
#include "../../include/oal.h"

using namespace oal;

static __device__ __align__(256) double g_noalloc_partials[OAL_NOALLOC_MAX_BLOCKS * 4];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch[kMaxDevices] = {};

// Per-block FP64 totals of the fluid cells; the obstacle array (uint8, 512 per block) or null.
template <class S, class R>
__global__ void k_mm_obstacle(const S* __restrict__ f, int64_t bst, int64_t kst, const uint8_t* __restrict__ obst,
                              double* __restrict__ part) {
  __shared__ double s[4][4];
  const int b = blockIdx.x, t = threadIdx.x;
  double m = 0, px = 0, py = 0, pz = 0;
  for (int cell = t; cell < kCells; cell += 128) {
    if (obst && obst[(int64_t)b * kCells + cell]) continue;
#pragma unroll
    for (int k = 0; k < kQ27; ++k) {
      const double v = (double)Codec<S>::dec(f[(int64_t)b * bst + k * kst + cell], R(q27_w(k)), R(1.0 / q27_w(k)));
      m += v; px += v * q27_cx(k); py += v * q27_cy(k); pz += v * q27_cz(k);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    m += __shfl_down_sync(0xffffffffu, m, o);
    px += __shfl_down_sync(0xffffffffu, px, o);
    py += __shfl_down_sync(0xffffffffu, py, o);
    pz += __shfl_down_sync(0xffffffffu, pz, o);
  }
  if ((t & 31) == 0) { s[0][t >> 5] = m; s[1][t >> 5] = px; s[2][t >> 5] = py; s[3][t >> 5] = pz; }
  __syncthreads();
  if (t < 4) part[4 * (int64_t)b + t] = ((s[t][0] + s[t][1]) + s[t][2]) + s[t][3];
}

// Fixed-order FP64 sum of n quadruples into out[4].
__global__ void k_mm_final(const double* __restrict__ part, int64_t n, double* __restrict__ out) {
  __shared__ double s[4][256];
  const int t = threadIdx.x;
  double a[4] = {0, 0, 0, 0};
  for (int64_t i = t; i < n; i += 256)
    for (int c = 0; c < 4; ++c) a[c] += part[4 * i + c];
  for (int c = 0; c < 4; ++c) s[c][t] = a[c];
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (t < w)
      for (int c = 0; c < 4; ++c) s[c][t] += s[c][t + w];
    __syncthreads();
  }
  if (t == 0)
    for (int c = 0; c < 4; ++c) out[c] = s[c][0];
}

template <class S, class R>
cudaError_t launch_mm(const void* f, int64_t bst, int64_t kst, const uint8_t* obst, int32_t nb, double* scratch,
                      double* out, cudaStream_t st) {
  k_mm_obstacle<S, R><<<nb, 128, 0, st>>>(static_cast<const S*>(f), bst, kst, obst, scratch);
  k_mm_final<<<1, 256, 0, st>>>(scratch, nb, out);
  return cudaGetLastError();
}

}  // namespace

// defined in level.cu
oal_status oal_internal_set_error(oal_status s, const char* msg);

extern "C" oal_status oal_mass_momentum_noalloc(const void* f, int32_t storage, int64_t f_block_stride,
                                                int64_t f_dir_stride, const uint8_t* obstacle, int32_t n_blocks,
                                                double* out, void* stream) {
  if (!f || !out) return oal_internal_set_error(OAL_E_INVALID_ARG, "f and out are required");
  if (n_blocks <= 0) return oal_internal_set_error(OAL_E_INVALID_ARG, "n_blocks must be positive");
  if (n_blocks > OAL_NOALLOC_MAX_BLOCKS) {
    char msg[160];
    snprintf(msg, sizeof msg, "n_blocks %d exceeds the fixed scratch of %d blocks", n_blocks, OAL_NOALLOC_MAX_BLOCKS);
    return oal_internal_set_error(OAL_E_TOO_LARGE, msg);
  }
  if (storage < OAL_STORE_F32 || storage > OAL_STORE_F64) return oal_internal_set_error(OAL_E_INVALID_ARG, "storage");
  if (f_block_stride < 512 || f_dir_stride < 512) return oal_internal_set_error(OAL_E_INVALID_ARG, "bad strides");
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return oal_internal_set_error(OAL_E_NO_DEVICE, "no current CUDA device");
  }
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch[dev]) {
      // once per device, with that device current: the device address of the file-scope array
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
      if (e != cudaSuccess || !p) {
        char msg[200];
        snprintf(msg, sizeof msg, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        return oal_internal_set_error(OAL_E_CUDA, msg);
      }
      g_scratch[dev] = static_cast<double*>(p);
    }
    scratch = g_scratch[dev];
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaErrorInvalidValue;
  switch (storage) {
    case OAL_STORE_F32: e = launch_mm<float, float>(f, f_block_stride, f_dir_stride, obstacle, n_blocks, scratch, out, st); break;
    case OAL_STORE_F16_DEV: e = launch_mm<__half, float>(f, f_block_stride, f_dir_stride, obstacle, n_blocks, scratch, out, st); break;
    case OAL_STORE_BF16_DEV: e = launch_mm<__nv_bfloat16, float>(f, f_block_stride, f_dir_stride, obstacle, n_blocks, scratch, out, st); break;
    case OAL_STORE_F64: e = launch_mm<double, double>(f, f_block_stride, f_dir_stride, obstacle, n_blocks, scratch, out, st); break;
  }
  if (e != cudaSuccess) {
    char msg[200];
    snprintf(msg, sizeof msg, "mass_momentum_noalloc launch: %s", cudaGetErrorString(e));
    return oal_internal_set_error(OAL_E_CUDA, msg);
  }
  return OAL_OK;
}
