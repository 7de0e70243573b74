// Allocation-free max |div u| (the DIVGCK_tg check) on caller-owned device
// arrays.
//
// Who needs it: hosts that may not call cudaMalloc at the point they want the
// check -- for example a solver that records its whole time step into its own
// CUDA graph (allocation is not allowed while a stream is being captured), or
// a host whose device memory is a fixed pool handed out by its own allocator
// so that a library allocating behind its back would break the budget.  Such
// a caller owns u, v, w and the output; this entry point brings no context
// and allocates nothing.
//
// The per-tile partial maxima live in one file-scope __device__ array of
// kNoAllocTiles doubles (512 KiB) that every GPU loading the library holds
// until the process exits.  Host code must not use the array's name as a
// device address (in host code it is only a stand-in symbol), so the first
// call on each device looks the address up with cudaGetSymbolAddress while
// that device is current and caches it.  Every call shares the array and it
// keeps the last call's tile maxima; each call writes every slot it later
// reads, so nothing needs clearing, but two calls whose kernels overlap on the
// GPU (different streams, or several host threads) race on it.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/chapsim.h"

// Largest channel served: 65,536 tiles of 32 x 8 (x, y) cells summed over the
// z planes, e.g. 256 x 256 x 256.  Larger ones get CHAPSIM_ERR_TOO_LARGE.
static constexpr int kNoAllocTiles = 65536;
static __device__ __align__(256) double g_divmax_partials[kNoAllocTiles];

namespace {

constexpr int kTX = 32, kTY = 8, kMaxDevices = 64;

double *g_partials_addr[kMaxDevices] = {nullptr};
std::mutex g_setup_mutex;

// Per-tile max |div u| of DIVGCK_tg (src/DIVGCK.f90:16-58), the arithmetic of
// the context path's reduction kernel.  Every tile writes its slot, so no
// slot needs clearing between calls.
__global__ void __launch_bounds__(kTX *kTY) k_divmax_tiles(const double *__restrict__ u, const double *__restrict__ v,
                                                          const double *__restrict__ w,
                                                          const double *__restrict__ dyfi, int nx, int ny, int nz,
                                                          double dxi, double dzi, double *partials) {
  __shared__ double sh[kTX * kTY / 32];
  const int i = blockIdx.x * kTX + threadIdx.x;
  const int j = blockIdx.y * kTY + threadIdx.y + 1;
  const int k = blockIdx.z;
  const int64_t sy = nx, sz = (int64_t)nx * (ny + 2);
  double val = 0.0;
  if (i < nx && j <= ny) {
    const int64_t c0 = i + sy * j + sz * k;
    const int ip = i + 1 == nx ? 0 : i + 1, kp = k + 1 == nz ? 0 : k + 1;
    const double dv = (u[c0 + (ip - i)] - u[c0]) * dxi + (v[c0 + sy] - v[c0]) * dyfi[j] +
                      (w[c0 + sz * (kp - k)] - w[c0]) * dzi;
    val = fabs(dv);
    if (dv != dv) val = __longlong_as_double(0x7ff0000000000000ll);  // NaN -> +inf
  }
  for (int o = 16; o > 0; o >>= 1) val = fmax(val, __shfl_xor_sync(0xffffffffu, val, o));
  const int tid = threadIdx.x + kTX * threadIdx.y;
  if ((tid & 31) == 0) sh[tid >> 5] = val;
  __syncthreads();
  if (tid == 0) {
    double m = 0.0;
    for (int q = 0; q < kTX * kTY / 32; ++q) m = fmax(m, sh[q]);
    partials[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = m;
  }
}

__global__ void __launch_bounds__(1024) k_divmax_final(const double *partials, int n, double *out) {
  __shared__ double sh[32];
  double m = 0.0;
  for (int t = threadIdx.x; t < n; t += blockDim.x) m = fmax(m, partials[t]);
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0.0;
    for (int q = 0; q < (int)(blockDim.x + 31) / 32; ++q) r = fmax(r, sh[q]);
    *out = r;
  }
}

}  // namespace

extern "C" int chapsim_divmax_noalloc(const double *u, const double *v, const double *w, const double *dyfi, int nx,
                                      int ny, int nz, double dxi, double dzi, double *out, void *stream) {
  if (!u || !v || !w || !dyfi || !out || nx < 1 || ny < 1 || nz < 1) return CHAPSIM_ERR_ARG;
  const int64_t tiles = (int64_t)((nx + kTX - 1) / kTX) * ((ny + kTY - 1) / kTY) * nz;
  if (tiles > kNoAllocTiles || nz > 65535) return CHAPSIM_ERR_TOO_LARGE;  // 65,535: grid z limit
  // an error left pending by the caller's own earlier work is not ours: leave
  // it in place for the caller and launch nothing
  if (cudaPeekAtLastError() != cudaSuccess) return CHAPSIM_ERR_CUDA;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return CHAPSIM_ERR_CUDA;
  }
  double *partials = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_partials_addr[dev]) {
      void *p = nullptr;
      if (cudaGetSymbolAddress(&p, g_divmax_partials) != cudaSuccess || !p) {
        cudaGetLastError();
        return CHAPSIM_ERR_CUDA;
      }
      g_partials_addr[dev] = static_cast<double *>(p);
    }
    partials = g_partials_addr[dev];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  dim3 grid((nx + kTX - 1) / kTX, (ny + kTY - 1) / kTY, nz);
  k_divmax_tiles<<<grid, dim3(kTX, kTY), 0, s>>>(u, v, w, dyfi, nx, ny, nz, dxi, dzi, partials);
  k_divmax_final<<<1, 1024, 0, s>>>(partials, (int)tiles, out);
  // no error was pending on entry, so one now comes from these two launches
  if (cudaGetLastError() != cudaSuccess) return CHAPSIM_ERR_CUDA;
  return CHAPSIM_OK;
}
