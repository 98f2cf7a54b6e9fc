// noalloc.cu — total stress of a contact set without any device allocation.
//
// Some callers cannot call cudaMalloc: code running inside a CUDA graph that is
// being captured (an allocation would break the capture), a host application
// that hands this library a fixed memory budget and owns every device buffer
// itself, or a real-time loop that must not take the allocator's locks.  For
// them, xdem_total_stress_noalloc computes the box stress of
// BaseWorld::updateTotalStress (BaseWorld.cpp:158-176),
//     sigma = sum_c F_c (x) b_c / area,
// from per-contact forces F and branch vectors b that the caller already holds
// on the device, with the same fixed-order tree reduction as the world path,
// but with its partial sums in a fixed array of this file instead of a buffer
// allocated per world.
//
// Limits and sharing:
//   - at most kNoallocMaxContacts contacts per call (larger calls are rejected);
//   - every GPU that loads the library holds the kNoallocMaxBlocks*4 doubles of
//     scratch until the process exits;
//   - all calls share that scratch: calls that may overlap on the GPU (different
//     streams, or one stream used from several host threads) race on it and
//     must be ordered by the caller;
//   - the array keeps the last call's partial sums; nothing needs clearing,
//     because every partial the final pass reads is written earlier in the
//     same call;
//   - the first call on a device looks up the scratch address for that device,
//     which needs that device to be current; make that first call before any
//     stream capture begins;
//   - the address is kept for the life of the process: a cudaDeviceReset (or
//     anything else that destroys the device's primary context) unloads the
//     array, so this entry point must not be called on that device after one;
//   - the status reports this call's own launches only (each launch's return
//     code), never an error an earlier, unrelated runtime call left behind.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/xdem_gpu.h"

namespace {

constexpr int kNoallocThreads = 256;
constexpr int kNoallocPerThread = 4;
constexpr int kNoallocPerBlock = kNoallocThreads * kNoallocPerThread;
constexpr int kNoallocMaxBlocks = 4096;
constexpr long long kNoallocMaxContacts = (long long)kNoallocMaxBlocks * kNoallocPerBlock;
constexpr int kMaxDevices = 64;

// block partial sums of the four stress components: 4 * 4096 doubles = 128 KiB
__device__ __align__(256) double g_stress_partials[4 * kNoallocMaxBlocks];

std::mutex g_addr_mutex;
double* g_addr[kMaxDevices] = {nullptr};

// device address of the scratch array for the current device
cudaError_t scratch_address(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_addr_mutex);
  if (!g_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_stress_partials);
    if (e != cudaSuccess) return e;
    g_addr[dev] = static_cast<double*>(p);
  }
  *out = g_addr[dev];
  return cudaSuccess;
}

// each block sums its contiguous run of contacts in a fixed tree
__global__ void __launch_bounds__(kNoallocThreads)
    k_noalloc_stress_blocks(long long nc, const double* __restrict__ fx, const double* __restrict__ fy,
                            const double* __restrict__ bx, const double* __restrict__ by,
                            double* partials, int nblocks) {
  __shared__ double sh[4][kNoallocThreads];
  const int t = threadIdx.x;
  const long long base = (long long)blockIdx.x * kNoallocPerBlock;
  double s[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
  for (int k = 0; k < kNoallocPerThread; ++k) {
    long long c = base + (long long)k * kNoallocThreads + t;
    if (c < nc) {
      // matrix2d::dyadic(force, branch) (MathMatrix2d.h:107-110)
      s[0] += fx[c] * bx[c];
      s[1] += fx[c] * by[c];
      s[2] += fy[c] * bx[c];
      s[3] += fy[c] * by[c];
    }
  }
  for (int q = 0; q < 4; ++q) sh[q][t] = s[q];
  __syncthreads();
  for (int off = kNoallocThreads / 2; off > 0; off >>= 1) {
    if (t < off)
      for (int q = 0; q < 4; ++q) sh[q][t] += sh[q][t + off];
    __syncthreads();
  }
  if (t == 0)
    for (int q = 0; q < 4; ++q) partials[(size_t)q * nblocks + blockIdx.x] = sh[q][0];
}

// one block sums the block partials in a fixed tree and divides by the area
__global__ void __launch_bounds__(kNoallocThreads)
    k_noalloc_stress_final(const double* partials, int nblocks, double area, double* stress) {
  __shared__ double sh[4][kNoallocThreads];
  const int t = threadIdx.x;
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  for (int b = t; b < nblocks; b += kNoallocThreads)
    for (int q = 0; q < 4; ++q) s[q] += partials[(size_t)q * nblocks + b];
  for (int q = 0; q < 4; ++q) sh[q][t] = s[q];
  __syncthreads();
  for (int off = kNoallocThreads / 2; off > 0; off >>= 1) {
    if (t < off)
      for (int q = 0; q < 4; ++q) sh[q][t] += sh[q][t + off];
    __syncthreads();
  }
  if (t == 0)
    for (int q = 0; q < 4; ++q) stress[q] = sh[q][0] / area;
}

}  // namespace

extern "C" int32_t xdem_total_stress_noalloc(int64_t ncontacts, const double* fx, const double* fy,
                                             const double* bx, const double* by, double area,
                                             double* stress, void* cuda_stream) {
  if (ncontacts < 0 || !stress || !(area > 0.0)) return XDEM_ERR_ARGUMENT;
  if (ncontacts > 0 && (!fx || !fy || !bx || !by)) return XDEM_ERR_ARGUMENT;
  if (ncontacts > kNoallocMaxContacts) return XDEM_ERR_CAPACITY;
  double* partials = nullptr;
  if (scratch_address(&partials) != cudaSuccess) return XDEM_ERR_CUDA;
  cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
  int nblocks = (int)((ncontacts + kNoallocPerBlock - 1) / kNoallocPerBlock);
  long long nc = ncontacts;
  // launched through cudaLaunchKernel, whose return code is this launch's own
  if (nblocks > 0) {
    void* args[] = {&nc, &fx, &fy, &bx, &by, &partials, &nblocks};
    if (cudaLaunchKernel((const void*)k_noalloc_stress_blocks, dim3(nblocks), dim3(kNoallocThreads),
                         args, 0, s) != cudaSuccess)
      return XDEM_ERR_CUDA;
  }
  // with no contacts the final pass reads no partials and writes zeros
  const double* cpartials = partials;
  void* fargs[] = {&cpartials, &nblocks, &area, &stress};
  if (cudaLaunchKernel((const void*)k_noalloc_stress_final, dim3(1), dim3(kNoallocThreads), fargs, 0,
                       s) != cudaSuccess)
    return XDEM_ERR_CUDA;
  return XDEM_OK;
}

extern "C" int64_t xdem_total_stress_noalloc_max_contacts(void) { return kNoallocMaxContacts; }
