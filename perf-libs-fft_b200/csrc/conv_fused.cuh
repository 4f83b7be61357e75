// Kernel template of the one-kernel Rader and Bluestein transforms
// (conv_fused.cu describes the algorithm); instantiated per algorithm in
// conv_fused_rader.cu and conv_fused_bluestein.cu so the two compile in
// parallel.
#pragma once
#include "kernels.h"
#include "pow2_stages.cuh"
#include "stockham_desc.h"

namespace plfft_b200 {

// table loads are issued kChunk at a time: with every load of a 32-element
// thread hoisted ahead of its use the kernel would exceed 128 registers
constexpr int kChunk = 8;
__device__ __forceinline__ void order_barrier() { asm volatile("" ::: "memory"); }

// Launch bounds: at most 256 threads per CTA (512 for m = 8192 at 16
// elements per thread), with MINB resident CTAs of 256 threads per SM,
// which caps the registers per thread at 65536 / (256 MINB).
template <int M, int E>
constexpr int conv_max_threads() { return M / E > 256 ? 512 : 256; }
template <int M, int E, int MINB>
constexpr int conv_min_blocks() { return M / E > 256 ? 1 : MINB; }

template <int M, int E, bool RADER, int MINB>
__global__ void __launch_bounds__(conv_max_threads<M, E>(), (conv_min_blocks<M, E, MINB>()))
    conv_fused_kernel(const ConvFusedLaunch L) {
  using P = P2<M, E>;
  constexpr int T = P::T;
  constexpr int PITCH = (spad_len_c(M) + 1) & ~1;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int grp = threadIdx.x / T;
  const int t = threadIdx.x - grp * T;
  const int64_t b = int64_t(blockIdx.x) * L.g + grp;
  const bool live = b < L.howmany;
  float2* buf = reinterpret_cast<float2*>(smraw) + grp * PITCH;
  const int n = L.n;
  auto sync = [&]() {
    if constexpr (T <= 32)
      __syncwarp();
    else
      __syncthreads();
  };

  // the member's n inputs enter through its shared-memory buffer (coalesced
  // global loads; Bluestein multiplies by the chirp on the way)
  const float2* src = L.in + b * L.idist;
  if (live)
    for (int j = t; j < n; j += T) {
      const float2 x = src[int64_t(j) * L.istride];
      buf[j] = RADER ? x : cmul(x, __ldg(L.chirp + j));
    }
  sync();
  float2 v[E];
  float2 x0 = make_float2(0.f, 0.f);
  if constexpr (RADER) {
    x0 = buf[0];
    // a_q = x[g^q], in chunks so the index loads do not all stay live
#pragma unroll
    for (int c = 0; c < E; c += kChunk) {
#pragma unroll
      for (int q = c; q < c + kChunk; ++q) {
        const int idx = t + T * q;
        v[q] = idx < n - 1 ? buf[__ldg(L.perm_in + idx)] : make_float2(0.f, 0.f);
      }
      order_barrier();
    }
  } else {
#pragma unroll
    for (int q = 0; q < E; ++q) {
      const int idx = t + T * q;
      v[q] = idx < n ? buf[idx] : make_float2(0.f, 0.f);
    }
  }

  // forward FFT_M (natural order in, natural order out: v[q] = A[t + T q])
  st_bfly<T, E, P::radix(0), 1, 0, -1>(v, t, L.tw);
  Stages<M, E, -1, 1>::run(v, t, buf, L.tw, sync);
  const float2 a0 = v[0];  // A[0] on thread t = 0
#pragma unroll
  for (int c = 0; c < E; c += kChunk) {
#pragma unroll
    for (int q = c; q < c + kChunk; ++q) v[q] = cmul(v[q], __ldg(L.spec + t + T * q));
    order_barrier();
  }
  // the inverse uses the same twiddle and exchange addresses as the forward
  // pass: opaque copies of the thread index and table pointer (tied to the
  // data) make the compiler recompute them instead of holding every address
  // of the forward pass live across it, which spilled registers
  int t2 = t;
  const float2* tw2 = L.tw;
  asm volatile("mov.b32 %0, %0;" : "+r"(t2) : "f"(v[E - 1].x));
  asm volatile("mov.b64 %0, %0;" : "+l"(tw2) : "f"(v[E - 1].y));
  st_bfly<T, E, P::radix(0), 1, 0, 1>(v, t2, tw2);
  Stages<M, E, 1, 1>::run(v, t2, buf, tw2, sync);

  // the outputs leave through the buffer too (Rader: inverse permutation)
  sync();  // the last exchange is fully read before the buffer is reused
  if constexpr (RADER) {
#pragma unroll
    for (int c = 0; c < E; c += kChunk) {
#pragma unroll
      for (int q = c; q < c + kChunk; ++q) {
        const int idx = t + T * q;
        if (idx < n - 1) buf[__ldg(L.perm_out + idx)] = cadd(x0, v[q]);
      }
      order_barrier();
    }
    if (t == 0) buf[0] = cadd(x0, a0);
  } else {
#pragma unroll
    for (int q = 0; q < E; ++q) {
      const int idx = t + T * q;
      if (idx < n) buf[idx] = v[q];
    }
  }
  sync();
  const float s = L.scale;
  float2* dst = L.out + b * L.odist;
  if (live)
    for (int j = t; j < n; j += T) {
      const float2 y = RADER ? buf[j] : cmul(buf[j], __ldg(L.chirp + j));
      dst[int64_t(j) * L.ostride] = cscale(y, s);
    }
}

template <int M, int E, bool RADER, int MINB>
cudaError_t run_conv_fused(const ConvFusedLaunch& L, cudaStream_t st) {
  auto* k = conv_fused_kernel<M, E, RADER, MINB>;
  const int threads = (M / E) * L.g;
  if (threads > conv_max_threads<M, E>() || L.g < 1) return cudaErrorInvalidValue;
  const int smem = conv_fused_smem_bytes(M, L.g);
  cudaError_t e = ensure_dynamic_smem(reinterpret_cast<const void*>(k), smem);
  if (e != cudaSuccess) return e;
  const int64_t grid = (L.howmany + L.g - 1) / L.g;
  k<<<dim3(unsigned(grid)), dim3(threads), smem, st>>>(L);
  return cudaGetLastError();
}

// Instantiated shapes (elements per thread e, register budget minb), the
// measured best first for each m:
//   m <= 512: (16, 3);  m = 1024: (32, 2), (16, 3);  m = 2048: (16, 3), (32, 2);
//   m = 4096: (16, 4), (16, 3), (32, 2);  m = 8192: (32, 2)
template <bool RADER>
cudaError_t launch_conv_fused_alg(int m, int e, int minb, const ConvFusedLaunch& L, cudaStream_t st) {
  const int key = e * 10 + minb;
  switch (m) {
    case 64: return key == 163 ? run_conv_fused<64, 16, RADER, 3>(L, st) : cudaErrorInvalidValue;
    case 128: return key == 163 ? run_conv_fused<128, 16, RADER, 3>(L, st) : cudaErrorInvalidValue;
    case 256: return key == 163 ? run_conv_fused<256, 16, RADER, 3>(L, st) : cudaErrorInvalidValue;
    case 512: return key == 163 ? run_conv_fused<512, 16, RADER, 3>(L, st) : cudaErrorInvalidValue;
    case 1024:
      if (key == 322) return run_conv_fused<1024, 32, RADER, 2>(L, st);
      return key == 163 ? run_conv_fused<1024, 16, RADER, 3>(L, st) : cudaErrorInvalidValue;
    case 2048:
      if (key == 163) return run_conv_fused<2048, 16, RADER, 3>(L, st);
      return key == 322 ? run_conv_fused<2048, 32, RADER, 2>(L, st) : cudaErrorInvalidValue;
    case 4096:
      if (key == 164) return run_conv_fused<4096, 16, RADER, 4>(L, st);
      if (key == 163) return run_conv_fused<4096, 16, RADER, 3>(L, st);
      return key == 322 ? run_conv_fused<4096, 32, RADER, 2>(L, st) : cudaErrorInvalidValue;
    case 8192: return key == 322 ? run_conv_fused<8192, 32, RADER, 2>(L, st) : cudaErrorInvalidValue;
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace plfft_b200
