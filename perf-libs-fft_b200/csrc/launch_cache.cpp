// Per-device caches for launch-time queries: a kernel's dynamic shared
// memory limit is raised once (to the largest size asked for so far) and
// occupancy answers are remembered, so repeated executions of a plan issue
// only the kernel launches themselves.
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <tuple>

#include "kernels.h"

namespace plfft_b200 {

namespace {
std::mutex g_mu;
std::map<std::pair<int, const void*>, int> g_smem;                  // (device, kernel) -> limit set
std::map<std::tuple<int, const void*, int, int>, int> g_occupancy;  // (device, kernel, threads, smem)
}  // namespace

cudaError_t ensure_dynamic_smem(const void* kernel, int bytes) {
  if (bytes <= 32 * 1024) return cudaSuccess;  // room for static shared memory below the default 48 KB
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(g_mu);
  int& have = g_smem[{dev, kernel}];
  if (have >= bytes) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) have = bytes;
  return e;
}

cudaError_t cached_blocks_per_sm(const void* kernel, int threads, int smem, int* blocks) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    auto it = g_occupancy.find({dev, kernel, threads, smem});
    if (it != g_occupancy.end()) {
      *blocks = it->second;
      return cudaSuccess;
    }
  }
  e = ensure_dynamic_smem(kernel, smem);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, kernel, threads, smem);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(g_mu);
  g_occupancy[{dev, kernel, threads, smem}] = *blocks;
  return cudaSuccess;
}

}  // namespace plfft_b200
