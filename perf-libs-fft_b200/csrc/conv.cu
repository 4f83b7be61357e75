// Rader and Bluestein convolution kernels (elementwise passes around the
// length-M C2C plans that do the convolution).
//
// Bluestein (reference src/planner/strategies/bluestein.hpp:37-240): with
// w_k = exp(dir * i pi (k^2 mod 2N) / N),
//   a_j = x_j w_j (j < N, zero to M),  A = FFT_M(a),  A *= B,
//   c = IFFT_M(A),  y_k = c_k w_k,
// where B = FFT_M(b)/M, b_m = conj(w_m) wrapped cyclically (|m| < N).
// Rader (reference src/planner/strategies/rader.hpp:36-254, generator
// src/rader_generator.cpp:13-33): for prime P with generator g,
//   a_q = x[g^q mod P],  A = FFT_{P-1}(a),  A0 = A[0] = sum_{j>0} x_j,
//   A *= B,  c = IFFT_{P-1}(A),  y[g^{-m} mod P] = x_0 + c_m,  y_0 = x_0 + A0,
// with B = FFT_{P-1}(exp(dir * 2 pi i g^{-m} / P)) / (P-1).
#include <algorithm>

#include "kernels.h"
#include "stockham.cuh"

namespace plfft_b200 {

__global__ void __launch_bounds__(256) bs_pre(const ConvLaunch L, int64_t m0, int64_t cnt) {
  const int64_t n = L.n, m = L.m;
  const int64_t total = cnt * m;
  const bool small = total < (int64_t(1) << 31);
  for (int64_t f = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; f < total; f += int64_t(gridDim.x) * blockDim.x) {
    const int64_t bl = flat_div(f, m, small);
    const int64_t j = f - bl * m;
    float2 z = make_float2(0.f, 0.f);
    if (j < n) z = cmul(L.in[(m0 + bl) * L.idist + j * L.istride], L.chirp[j]);
    L.work[f] = z;
  }
}

// work *= spec (per member), optionally saving element 0 first (Rader)
__global__ void __launch_bounds__(256) conv_mul(const ConvLaunch L, int64_t cnt, int save0) {
  const int64_t m = L.m;
  const int64_t total = cnt * m;
  const bool small = total < (int64_t(1) << 31);
  for (int64_t f = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; f < total; f += int64_t(gridDim.x) * blockDim.x) {
    const int64_t bl = flat_div(f, m, small);
    const int64_t k = f - bl * m;
    const float2 a = L.work[f];
    if (save0 && k == 0) L.sum0[bl] = a;
    L.work[f] = cmul(a, L.spec[k]);
  }
}

__global__ void __launch_bounds__(256) bs_post(const ConvLaunch L, int64_t m0, int64_t cnt) {
  const int64_t n = L.n, m = L.m;
  const int64_t total = cnt * n;
  const bool small = total < (int64_t(1) << 31);
  const float s = L.scale;
  for (int64_t f = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; f < total; f += int64_t(gridDim.x) * blockDim.x) {
    const int64_t bl = flat_div(f, n, small);
    const int64_t k = f - bl * n;
    const float2 y = cmul(L.work[bl * m + k], L.chirp[k]);
    L.out[(m0 + bl) * L.odist + k * L.ostride] = cscale(y, s);
  }
}

__global__ void __launch_bounds__(256) rd_pre(const ConvLaunch L, int64_t m0, int64_t cnt) {
  const int64_t m = L.m;  // P - 1
  const int64_t total = cnt * m;
  const bool small = total < (int64_t(1) << 31);
  for (int64_t f = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; f < total; f += int64_t(gridDim.x) * blockDim.x) {
    const int64_t bl = flat_div(f, m, small);
    const int64_t q = f - bl * m;
    L.work[f] = L.in[(m0 + bl) * L.idist + int64_t(L.perm_in[q]) * L.istride];
  }
}

__global__ void __launch_bounds__(256) rd_post(const ConvLaunch L, int64_t m0, int64_t cnt) {
  const int64_t m = L.m;
  const int64_t total = cnt * m;
  const bool small = total < (int64_t(1) << 31);
  const float s = L.scale;
  for (int64_t f = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; f < total; f += int64_t(gridDim.x) * blockDim.x) {
    const int64_t bl = flat_div(f, m, small);
    const int64_t q = f - bl * m;
    const int64_t b = m0 + bl;
    const float2 x0 = L.in[b * L.idist];
    float2* y = L.out + b * L.odist;
    y[int64_t(L.perm_out[q]) * L.ostride] = cscale(cadd(x0, L.work[f]), s);
    if (q == 0) y[0] = cscale(cadd(x0, L.sum0[bl]), s);
  }
}

static unsigned grid_for(int64_t total) {
  return unsigned(std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, 148 * 16)));
}

cudaError_t launch_conv(int step, const ConvLaunch& L, int64_t m0, int64_t cnt, cudaStream_t st) {
  switch (step) {
    case CONV_BS_PRE: bs_pre<<<grid_for(cnt * L.m), 256, 0, st>>>(L, m0, cnt); break;
    case CONV_MUL: conv_mul<<<grid_for(cnt * L.m), 256, 0, st>>>(L, cnt, 0); break;
    case CONV_MUL_SAVE0: conv_mul<<<grid_for(cnt * L.m), 256, 0, st>>>(L, cnt, 1); break;
    case CONV_BS_POST: bs_post<<<grid_for(cnt * L.n), 256, 0, st>>>(L, m0, cnt); break;
    case CONV_RD_PRE: rd_pre<<<grid_for(cnt * L.m), 256, 0, st>>>(L, m0, cnt); break;
    case CONV_RD_POST: rd_post<<<grid_for(cnt * L.m), 256, 0, st>>>(L, m0, cnt); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace plfft_b200
