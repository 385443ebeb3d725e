// Weighted inner product that allocates no device memory.
//
// Some host applications cannot let a library call cudaMalloc: a serving
// process that hands the whole device memory to its own pool at start-up
// and runs under a fixed HBM budget, or a time-stepping loop that must never
// hit cudaMalloc's implicit device-wide synchronisation.  This entry point
// computes the same quantity as ssg_global_dot_product -- sum over the
// L-vector of (x * w) * y with w = 1/multiplicity, global_dot_product in the
// reference (src/global.c:270-282) -- from caller-owned device buffers, and
// keeps its block partial sums in a file-scope __device__ array instead of a
// context workspace.
//
// The array holds SSG_NOALLOC_MAX_BLOCKS doubles (512 KiB) on every GPU that
// loads the library, until the process exits.  One block covers
// SSG_NOALLOC_POINTS_PER_BLOCK points, so the entry point accepts at most
// SSG_NOALLOC_MAX_BLOCKS * SSG_NOALLOC_POINTS_PER_BLOCK = 134,217,728
// points and rejects larger sizes with SSG_ERR_ARG.
//
// All calls in the process share that one array, and each call leaves its
// partial sums in it.  Every call writes every partial slot it later reads,
// so nothing needs clearing, but two calls whose kernels overlap on the GPU
// (different streams, no ordering between them) race on the array and must
// not be issued.
//
// The first call on a device looks up the array's device address with
// cudaGetSymbolAddress (once per device, with that device current); make
// that first call before any stream capture on the device.  The address is
// cached for the life of the process: a cudaDeviceReset unloads the module,
// and calls after it are not supported.
//
// Every pointer must be device memory of the current device (or managed
// memory); host memory and another GPU's memory are rejected with
// SSG_ERR_ARG.
#include <cuda_runtime.h>

#include <cstddef>
#include <mutex>

#include "ssenss_b200.h"

#define SSG_NOALLOC_THREADS 256
#define SSG_NOALLOC_PER_THREAD 8
#define SSG_NOALLOC_POINTS_PER_BLOCK (SSG_NOALLOC_THREADS * SSG_NOALLOC_PER_THREAD)
#define SSG_NOALLOC_MAX_BLOCKS 65536
#define SSG_NOALLOC_MAX_DEVICES 64

// block partial sums of every call (device memory, fixed size)
static __device__ __align__(256) double g_noalloc_partials[SSG_NOALLOC_MAX_BLOCKS];

namespace {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// one partial per block over a fixed slice of SSG_NOALLOC_POINTS_PER_BLOCK
// points, fixed reduction order (deterministic)
__global__ void __launch_bounds__(SSG_NOALLOC_THREADS)
k_wdot_partials(size_t n, const double* __restrict__ x, const double* __restrict__ y,
                const double* __restrict__ w, double* __restrict__ partials) {
  __shared__ double s[SSG_NOALLOC_THREADS / 32];
  const size_t base = (size_t)blockIdx.x * SSG_NOALLOC_POINTS_PER_BLOCK;
  double v = 0.0;
#pragma unroll
  for (int r = 0; r < SSG_NOALLOC_PER_THREAD; ++r) {
    const size_t q = base + (size_t)r * SSG_NOALLOC_THREADS + threadIdx.x;
    if (q < n) v += (x[q] * w[q]) * y[q];
  }
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = threadIdx.x < SSG_NOALLOC_THREADS / 32 ? s[threadIdx.x] : 0.0;
    t = warp_sum(t);
    if (threadIdx.x == 0) partials[blockIdx.x] = t;
  }
}

// sum of the nblk partials by one block, fixed order; result to the caller
__global__ void __launch_bounds__(SSG_NOALLOC_THREADS)
k_wdot_final(int nblk, const double* __restrict__ partials, double* __restrict__ result) {
  __shared__ double s[SSG_NOALLOC_THREADS / 32];
  double v = 0.0;
  for (int b = threadIdx.x; b < nblk; b += SSG_NOALLOC_THREADS) v += partials[b];
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = threadIdx.x < SSG_NOALLOC_THREADS / 32 ? s[threadIdx.x] : 0.0;
    t = warp_sum(t);
    if (threadIdx.x == 0) *result = t;
  }
}

std::mutex g_mu;
double* g_partials_addr[SSG_NOALLOC_MAX_DEVICES] = {};

// true for device memory of GPU `dev` (the current device) and for managed
// memory; false for host memory and for another GPU's device memory, which a
// kernel on `dev` would reach only through peer access, if at all
bool on_device(const void* p, int dev) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (a.type == cudaMemoryTypeManaged) return true;
  return a.type == cudaMemoryTypeDevice && a.device == dev;
}

// device address of g_noalloc_partials on device `dev`, the current device
// (looked up once per device; the cached address does not survive a
// cudaDeviceReset, after which the module loads anew)
ssg_status partials_address(int dev, double** out) {
  if (dev < 0 || dev >= SSG_NOALLOC_MAX_DEVICES) return SSG_ERR_ARG;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_partials_addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_partials) != cudaSuccess || !p) {
      cudaGetLastError();
      return SSG_ERR_CUDA;
    }
    g_partials_addr[dev] = static_cast<double*>(p);
  }
  *out = g_partials_addr[dev];
  return SSG_OK;
}

}  // namespace

extern "C" ssg_status ssg_weighted_dot_noalloc(const double* x, const double* y,
                                               const double* w, size_t n, double* result,
                                               void* cuda_stream) {
  if (!x || !y || !w || !result) return SSG_ERR_ARG;
  const size_t max_points = (size_t)SSG_NOALLOC_MAX_BLOCKS * SSG_NOALLOC_POINTS_PER_BLOCK;
  if (n > max_points) return SSG_ERR_ARG;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return SSG_ERR_CUDA;
  }
  if (!on_device(x, dev) || !on_device(y, dev) || !on_device(w, dev) ||
      !on_device(result, dev))
    return SSG_ERR_ARG;
  cudaStream_t s = (cudaStream_t)cuda_stream;
  if (n == 0) {
    if (cudaMemsetAsync(result, 0, sizeof(double), s) != cudaSuccess) return SSG_ERR_CUDA;
    return SSG_OK;
  }
  double* partials = nullptr;
  const ssg_status st = partials_address(dev, &partials);
  if (st != SSG_OK) return st;
  const int nblk = (int)((n + SSG_NOALLOC_POINTS_PER_BLOCK - 1) / SSG_NOALLOC_POINTS_PER_BLOCK);
  k_wdot_partials<<<nblk, SSG_NOALLOC_THREADS, 0, s>>>(n, x, y, w, partials);
  k_wdot_final<<<1, SSG_NOALLOC_THREADS, 0, s>>>(nblk, partials, result);
  if (cudaGetLastError() != cudaSuccess) return SSG_ERR_CUDA;
  return SSG_OK;
}
