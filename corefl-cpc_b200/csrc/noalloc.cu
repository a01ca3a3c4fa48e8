// cb2_min_dt_noalloc: the global minimum of a per-node time-step array, for callers that may
// not allocate device memory.
//
// Some embedding codes hand every byte of device memory to their own pool before the solver
// starts and forbid cudaMalloc afterwards; others cannot afford the device-wide
// synchronisation that cudaFree implies while other streams run.  Such a caller can still
// reduce the local CFL steps that local_time_step writes into dt_local: this entry point
// takes the array and returns its minimum without allocating anything.
//
// The per-CTA partial minima live in g_noalloc_partials, a file-scope __device__ array of
// CB2_NOALLOC_MAX_PARTIALS doubles that every GPU loading the library keeps until the process
// exits.  Host code must not use the array's name as a device address, so the address is
// resolved with cudaGetSymbolAddress once per device, on the first call made with that device
// current; that first call should therefore come before any stream capture.  The resolved
// address is kept per device ordinal for the life of the process: it assumes the device's primary
// context (the runtime's own) and no cudaDeviceReset in between, after which the array would live
// at a new address.  All calls share the array, so calls whose kernels overlap on the GPU race
// with each other.
#include <mutex>
#include "common.cuh"
#include "launch.h"

namespace cb2 {
namespace {

constexpr int kNaThreads = 256;
constexpr int kNaPerThread = 8;                                // elements per thread
constexpr long long kNaPerCta = (long long)kNaThreads * kNaPerThread;
constexpr int kNaMaxDevices = 64;
// every n the entry point accepts must fit its partial minima in the array
static_assert(CB2_NOALLOC_MAX_NODES <= (long long)CB2_NOALLOC_MAX_PARTIALS * kNaPerCta,
              "CB2_NOALLOC_MAX_NODES exceeds the partial-minimum capacity");

static __device__ __align__(256) double g_noalloc_partials[CB2_NOALLOC_MAX_PARTIALS];

std::mutex g_na_mutex;
double *g_na_addr[kNaMaxDevices] = {};

__device__ __forceinline__ double na_warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ double na_block_min(double v) {
  __shared__ double sw[kNaThreads / 32];
  v = na_warp_min(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sw[wid] = v;
  __syncthreads();
  if (wid == 0) {
    v = lane < kNaThreads / 32 ? sw[lane] : 1e+6;
    v = na_warp_min(v);
  }
  return v;
}

// One partial minimum per CTA over kNaPerCta consecutive elements; every thread starts from
// 1e+6 as min_of_arr does (src/TimeAdvanceFunc.cu:152).
__global__ void __launch_bounds__(kNaThreads) k_na_partial(const double *src, long long n, double *partial) {
  double v = 1e+6;
  const long long base = (long long)blockIdx.x * kNaPerCta + threadIdx.x;
#pragma unroll
  for (int m = 0; m < kNaPerThread; ++m) {
    const long long e = base + (long long)m * kNaThreads;
    if (e < n) v = fmin(v, src[e]);
  }
  v = na_block_min(v);
  if (threadIdx.x == 0) partial[blockIdx.x] = v;
}

__global__ void __launch_bounds__(kNaThreads) k_na_final(const double *partial, int n_partial, double *out) {
  double v = 1e+6;
  for (int t = threadIdx.x; t < n_partial; t += kNaThreads) v = fmin(v, partial[t]);
  v = na_block_min(v);
  if (threadIdx.x == 0) *out = v;
}

// Device address of g_noalloc_partials for the current device, resolved once per device.
int na_scratch(double **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_cuda_error(e);
    return CB2_ERR_CUDA;
  }
  if (dev < 0 || dev >= kNaMaxDevices) return CB2_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_na_mutex);
  if (!g_na_addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_partials);
    if (e != cudaSuccess) {
      set_cuda_error(e);
      return CB2_ERR_CUDA;
    }
    g_na_addr[dev] = static_cast<double *>(p);
  }
  *out = g_na_addr[dev];
  return CB2_OK;
}

}  // namespace
}  // namespace cb2

extern "C" int cb2_min_dt_noalloc(const double *dt_local, long long n, double *dt_min, void *stream) {
  using namespace cb2;
  if (!dt_local || !dt_min || n < 1) return CB2_ERR_INVALID;
  if (n > (long long)CB2_NOALLOC_MAX_NODES) return CB2_ERR_INVALID;  // beyond the scratch capacity
  double *partial = nullptr;
  CB2_TRY(na_scratch(&partial));
  const int n_partial = (int)((n + kNaPerCta - 1) / kNaPerCta);
  cudaStream_t s = (cudaStream_t)stream;
  k_na_partial<<<n_partial, kNaThreads, 0, s>>>(dt_local, n, partial);
  CB2_TRY(check_launch());
  k_na_final<<<1, kNaThreads, 0, s>>>(partial, n_partial, dt_min);
  return check_launch();
}
