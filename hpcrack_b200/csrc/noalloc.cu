// Allocation-free entry point: the d_max / delta_d_max reduction of caller-owned device arrays,
// with its block partials in a fixed, statically allocated device array instead of memory the
// library or the caller allocates.
//
// Who needs it: code that must not call cudaMalloc / cudaFree while it runs - a host program whose
// device memory is owned by a pool allocator that forbids foreign allocations, code between the
// steps of a time-critical loop where cudaMalloc's implicit device synchronisation is not
// acceptable, or a caller that simply has no allocation rights on the device it is handed.
//
// Contract (see include/hpcrack.h, hpc_dmax_noalloc):
//   * scratch: g_dmax_scratch, kDmaxMaxBlocks block partials (2 doubles each) plus a completion
//     counter, 1 MiB per device, resident on every device that loads the library until exit;
//   * n is limited to kDmaxMaxBlocks * kDmaxPerBlock = 134,217,728 values (a 512^3-node level);
//     larger n is rejected with HPC_ERR_ARG;
//   * the first call on a device looks up the scratch address with cudaGetSymbolAddress, with that
//     device current, and checks the result; later calls on that device reuse the address.  With
//     lazy module loading (the CUDA 12 default) that first lookup can be what loads this library's
//     device code and places the scratch, so the first call may allocate and synchronise: make one
//     warm-up call (or any other call of this library on that device) before a region that must
//     not allocate, and before any stream capture.  The cached address does not survive
//     cudaDeviceReset (the caller must not reset a device it keeps using this library on);
//   * every call shares the scratch: calls that overlap on the GPU race.  The counter is cleared
//     by each call before its kernel, so a call never depends on what the previous call left.
#include <cuda_runtime.h>

#include <atomic>

#include "device_common.cuh"
#include "internal.h"

namespace hpc {
namespace {

constexpr int kDmaxThreads = 256;
constexpr int kDmaxPerThread = 8;
constexpr long long kDmaxPerBlock = (long long)kDmaxThreads * kDmaxPerThread;  // 2048 values
constexpr long long kDmaxMaxBlocks = 65536;
constexpr long long kDmaxMaxN = kDmaxMaxBlocks * kDmaxPerBlock;                // 134,217,728
constexpr long long kScratchDoubles = 2 * kDmaxMaxBlocks + 32;                 // partials + counter

static __device__ __align__(256) double g_dmax_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
// Per-device scratch address.  Two threads making their first call on one device at once both look
// the address up and store the same value; the atomic makes that race well defined.
std::atomic<double*> g_scratch_ptr[kMaxDevices] = {};

// out[0] = max(0, max(d - d_old)), out[1] = max(0, max(d)) (phase_field_max_search.cpp:17-53).
__global__ void __launch_bounds__(kDmaxThreads) dmax_noalloc_kernel(const double* d, const double* d_old, long long n,
                                                                     double* scratch, double* out) {
  double* partials = scratch;  // [2][gridDim.x]
  unsigned int* counter = reinterpret_cast<unsigned int*>(scratch + 2 * kDmaxMaxBlocks);
  __shared__ double s_dd[kDmaxThreads / 32], s_dm[kDmaxThreads / 32];
  __shared__ int s_last;
  double dd = 0.0, dm = 0.0;
  const long long base = (long long)blockIdx.x * kDmaxPerBlock;
#pragma unroll
  for (int q = 0; q < kDmaxPerThread; ++q) {
    const long long i = base + (long long)q * kDmaxThreads + threadIdx.x;
    if (i < n) {
      const double v = d[i];
      dd = fmax(dd, v - d_old[i]);
      dm = fmax(dm, v);
    }
  }
  dd = warp_max(dd);
  dm = warp_max(dm);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    s_dd[warp] = dd;
    s_dm[warp] = dm;
  }
  __syncthreads();
  if (warp == 0) {
    dd = lane < kDmaxThreads / 32 ? s_dd[lane] : 0.0;
    dm = lane < kDmaxThreads / 32 ? s_dm[lane] : 0.0;
    dd = warp_max(dd);
    dm = warp_max(dm);
    if (lane == 0) {
      partials[blockIdx.x] = dd;
      partials[kDmaxMaxBlocks + blockIdx.x] = dm;
      __threadfence();
      s_last = atomicAdd(counter, 1u) == gridDim.x - 1u;
    }
  }
  __syncthreads();
  if (s_last && warp == 0) {
    __threadfence();
    dd = 0.0;
    dm = 0.0;
    for (unsigned b = lane; b < gridDim.x; b += 32) {
      dd = fmax(dd, __ldcg(partials + b));
      dm = fmax(dm, __ldcg(partials + kDmaxMaxBlocks + b));
    }
    dd = warp_max(dd);
    dm = warp_max(dm);
    if (lane == 0) {
      out[0] = dd;
      out[1] = dm;
      *counter = 0u;
    }
  }
}

}  // namespace
}  // namespace hpc

extern "C" int hpc_dmax_noalloc(const double* d, const double* d_old, long long n, double* out, void* stream) {
  using namespace hpc;
  if (!d || !d_old || !out) {
    set_error("hpc_dmax_noalloc: null pointer");
    return HPC_ERR_ARG;
  }
  if (n < 1 || n > kDmaxMaxN) {
    set_error("hpc_dmax_noalloc: n must be in [1, 134217728] (the fixed scratch holds 65536 block partials)");
    return HPC_ERR_ARG;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "hpc_dmax_noalloc: cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("hpc_dmax_noalloc: device index beyond the supported range");
    return HPC_ERR_ARG;
  }
  double* scratch = g_scratch_ptr[dev].load(std::memory_order_acquire);
  if (!scratch) {  // one-time set-up on this device (the current one)
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_dmax_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "hpc_dmax_noalloc: cudaGetSymbolAddress");
    scratch = static_cast<double*>(p);
    g_scratch_ptr[dev].store(scratch, std::memory_order_release);
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  e = cudaMemsetAsync(scratch + 2 * kDmaxMaxBlocks, 0, sizeof(unsigned int), s);
  if (e != cudaSuccess) return cuda_fail(e, "hpc_dmax_noalloc: clearing the counter");
  const unsigned blocks = (unsigned)((n + kDmaxPerBlock - 1) / kDmaxPerBlock);
  dmax_noalloc_kernel<<<blocks, kDmaxThreads, 0, s>>>(d, d_old, n, scratch, out);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "hpc_dmax_noalloc: launch");
  return HPC_OK;
}
