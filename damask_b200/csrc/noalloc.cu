// Volume average of a device-resident 9-component field without any allocation.
//
// Who needs it: a host that must not allocate device memory after set-up -- for
// example a solver loop that runs inside a fixed memory arena handed out by its own
// framework, or a real-time / budgeted loop in which a device allocation (and the
// device-wide synchronisation cudaMalloc/cudaFree can imply) is not allowed.  Such
// a caller owns its field in device memory and only wants <f> back.
//
// The per-block partial sums, which the context-based path keeps in memory the
// context allocated, live here in one file-scope device array that every GPU
// loading the library holds until the process exits.
#include "../../include/damask_b200.h"

#include <cuda_runtime.h>

#include <string>

namespace dmk {
void set_last_error(const std::string& msg);   // context.cu: text returned by dmk_last_error()
}

namespace {

constexpr int NA_THREADS = 256;
constexpr int NA_VOXELS_PER_THREAD = 4;
constexpr int64_t NA_VOXELS_PER_BLOCK = int64_t(NA_THREADS) * NA_VOXELS_PER_THREAD;
constexpr int NA_MAX_BLOCKS = 16384;                       // => at most 16,777,216 voxels (256^3)
constexpr int64_t NA_MAX_VOXELS = NA_VOXELS_PER_BLOCK * NA_MAX_BLOCKS;

// 9 partial sums per block, then the 9 results: 147,465 doubles = 1.13 MiB per GPU
static __device__ __align__(256) double g_mean_scratch[NA_MAX_BLOCKS * 9 + 9];

__global__ void __launch_bounds__(NA_THREADS)
na_partial_kernel(const double* __restrict__ f, int64_t n, double* __restrict__ part) {
  __shared__ double red[9][NA_THREADS / 32];
  double s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  const int64_t base = int64_t(blockIdx.x) * NA_VOXELS_PER_BLOCK + threadIdx.x;
#pragma unroll
  for (int r = 0; r < NA_VOXELS_PER_THREAD; ++r) {
    const int64_t v = base + int64_t(r) * NA_THREADS;
    if (v < n)
#pragma unroll
      for (int k = 0; k < 9; ++k) s[k] += f[k * n + v];
  }
#pragma unroll
  for (int k = 0; k < 9; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s[k] += __shfl_down_sync(0xffffffffu, s[k], o);
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int k = 0; k < 9; ++k) red[k][threadIdx.x >> 5] = s[k];
  __syncthreads();
  if (threadIdx.x < 9) {
    double t = 0.0;
    for (int w = 0; w < NA_THREADS / 32; ++w) t += red[threadIdx.x][w];
    part[int64_t(blockIdx.x) * 9 + threadIdx.x] = t;      // every call overwrites its slots
  }
}

__global__ void na_final_kernel(const double* __restrict__ part, int nblocks, double scale, double* __restrict__ out) {
  const int k = threadIdx.x;
  if (k >= 9) return;
  double t = 0.0;
  for (int b = 0; b < nblocks; ++b) t += part[int64_t(b) * 9 + k];
  out[k] = t * scale;
}

// Set-up, with the calling thread's current device: the device address of the array on that
// device.  It is looked up on every call (a table lookup once the library's device code is
// loaded on the device) rather than cached, so it stays right after the host resets a device.
int na_scratch(double** ptr) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0) {
    dmk::set_last_error(std::string("dmk_field_mean_noalloc: no current CUDA device: ") + cudaGetErrorString(e));
    return DMK_ERR_CUDA;
  }
  double* p = nullptr;
  e = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_mean_scratch);
  if (e != cudaSuccess || !p) {
    dmk::set_last_error(std::string("dmk_field_mean_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
    return DMK_ERR_CUDA;
  }
  *ptr = p;
  return 0;
}

}  // namespace

extern "C" {

int dmk_field_mean_noalloc(const double* field, int64_t n_voxels, double mean[9], void* stream) {
  if (!field || !mean) {
    dmk::set_last_error("dmk_field_mean_noalloc: null argument");
    return DMK_ERR_ARG;
  }
  if (n_voxels < 1 || n_voxels > NA_MAX_VOXELS) {
    dmk::set_last_error("dmk_field_mean_noalloc: n_voxels must be in [1, 16777216] (fixed scratch of 16384 blocks)");
    return DMK_ERR_ARG;
  }
  double* scratch = nullptr;
  if (int rc = na_scratch(&scratch)) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int nb = int((n_voxels + NA_VOXELS_PER_BLOCK - 1) / NA_VOXELS_PER_BLOCK);
  double* part = scratch;
  double* res = scratch + int64_t(NA_MAX_BLOCKS) * 9;
  na_partial_kernel<<<nb, NA_THREADS, 0, s>>>(field, n_voxels, part);
  na_final_kernel<<<1, 32, 0, s>>>(part, nb, 1.0 / double(n_voxels), res);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(mean, res, 9 * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    dmk::set_last_error(std::string("dmk_field_mean_noalloc: ") + cudaGetErrorString(e));
    return DMK_ERR_CUDA;
  }
  return 0;
}

}  // extern "C"
