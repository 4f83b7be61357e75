// FP16 data type: conversion passes around an FP32 schedule.
//
// The reference's FP16 plans take and return binary16 data
// (include/plfft.h:143-154, docs/plfft.md:244-255).  Here the caller's
// strided half data of a chunk of members is widened into a dense FP32
// chunk, transformed by the FP32 schedule, and rounded back to binary16
// (round to nearest even) into the caller's strided output.  Arithmetic is
// FP32 throughout, so the only rounding beyond the FP32 path is that of the
// output to half.
#include <cuda_fp16.h>

#include "kernels.h"

namespace plfft_b200 {

// dense[(b - m0) * n + k] <- half(src[b * dist + k * stride]), comps = 1
// (real) or 2 (complex) scalars per element
__global__ void __launch_bounds__(256) half_gather(const __half* __restrict__ src, float* __restrict__ dense,
                                                   int64_t m0, int64_t cnt, int64_t n, int64_t stride, int64_t dist,
                                                   int comps) {
  const int64_t total = cnt * n;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t b = i / n, k = i - b * n;
    const int64_t s = ((m0 + b) * dist + k * stride) * comps;
    if (comps == 2)
      reinterpret_cast<float2*>(dense)[i] = make_float2(__half2float(src[s]), __half2float(src[s + 1]));
    else
      dense[i] = __half2float(src[s]);
  }
}

// dst[b * dist + k * stride] <- half(dense[(b - m0) * n + k])
__global__ void __launch_bounds__(256) half_scatter(const float* __restrict__ dense, __half* __restrict__ dst,
                                                    int64_t m0, int64_t cnt, int64_t n, int64_t stride, int64_t dist,
                                                    int comps) {
  const int64_t total = cnt * n;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t b = i / n, k = i - b * n;
    const int64_t d = ((m0 + b) * dist + k * stride) * comps;
    if (comps == 2) {
      const float2 v = reinterpret_cast<const float2*>(dense)[i];
      dst[d] = __float2half_rn(v.x);
      dst[d + 1] = __float2half_rn(v.y);
    } else {
      dst[d] = __float2half_rn(dense[i]);
    }
  }
}

static unsigned grid_for(int64_t total) {
  const int64_t blocks = (total + 255) / 256;
  return unsigned(blocks < 148 * 16 ? (blocks > 0 ? blocks : 1) : 148 * 16);
}

cudaError_t launch_half_gather(const void* src, float* dense, int64_t m0, int64_t cnt, int64_t n, int64_t stride,
                               int64_t dist, int comps, cudaStream_t st) {
  half_gather<<<grid_for(cnt * n), 256, 0, st>>>(static_cast<const __half*>(src), dense, m0, cnt, n, stride, dist,
                                                 comps);
  return cudaGetLastError();
}

cudaError_t launch_half_scatter(const float* dense, void* dst, int64_t m0, int64_t cnt, int64_t n, int64_t stride,
                                int64_t dist, int comps, cudaStream_t st) {
  half_scatter<<<grid_for(cnt * n), 256, 0, st>>>(dense, static_cast<__half*>(dst), m0, cnt, n, stride, dist, comps);
  return cudaGetLastError();
}

}  // namespace plfft_b200
