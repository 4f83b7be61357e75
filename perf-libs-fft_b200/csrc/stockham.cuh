// Stockham autosort FFT engines for one or more transforms resident on chip.
//
// A length-N transform is a sequence of radix stages R_0, R_1, ... with
// Ns = R_0 * ... * R_{s-1} (the sub-transform length already done).  Stage s
// takes butterfly j in [0, N/R) from A[j + i*N/R] (i < R), multiplies input i
// by W_{Ns*R}^{(j mod Ns)*i}, applies DFT_R and writes output i to
//   B[(j / Ns) * Ns * R + (j mod Ns) + i * Ns].
// This is the GPU replacement of the reference's level chain
// (src/exec_compositor.cpp:18-50 ping-pongs between two n-sized buffers,
// level_ab_n / level_ac_t / level_ab_t apply one radix per level with the
// twiddle rows of src/generate_twiddles.hpp:72-136).  Here all levels of one
// transform run inside one CTA and exchange through shared memory.
//
// Twiddle table layout: stage s owns (R-1)*Ns entries at tw_off,
//   tw[tw_off + (i-1)*Ns + r] = exp(-2 pi i * r * i / (Ns*R))
// (forward sign; backward conjugates at use), so lanes with consecutive j
// read consecutive entries.
//
// Two engines:
//  * RegFFT<E>: each of T = N/E threads keeps E elements in registers.  The
//    first stage reads global memory directly and the last stage leaves the
//    result in registers, so an N = R0*R1 transform costs one shared-memory
//    exchange.  Requires every radix to divide E.
//  * smem_fft<MAXE>: general engine; a CTA holds C transforms in shared
//    memory and every stage is a read-all / barrier / write-all pass.
#pragma once
#include "codelets.cuh"
#include "stockham_desc.h"

namespace plfft_b200 {

// f / d for the flat element loops of the elementwise kernels: 32-bit
// division (a short sequence) when the loop's range fits 31 bits, which the
// 64 MB chunks of those kernels guarantee in practice
__device__ __forceinline__ int64_t flat_div(int64_t f, int64_t d, bool small) {
  return small ? int64_t(uint32_t(f) / uint32_t(d)) : f / d;
}

// shared-memory index padding: one spare complex every 16 (128 bytes)
__device__ __forceinline__ int spad(int p) { return p + (p >> 4); }

__device__ __forceinline__ int div_ns(int j, const Stage& s) {
  return s.ns_shift >= 0 ? (j >> s.ns_shift) : (j / s.ns);
}

// ===========================================================================
// Register engine
// ===========================================================================
template <int E, int R, int DIR>
__device__ __forceinline__ void reg_butterflies(float2 (&v)[E], int t, int T, const Stage& s,
                                                const float2* __restrict__ tw) {
  constexpr int M = E / R;
#pragma unroll
  for (int m = 0; m < M; ++m) {
    float2 x[R];
#pragma unroll
    for (int i = 0; i < R; ++i) x[i] = v[m + M * i];
    if (s.ns > 1) {
      const int j = t + T * m;
      const int r = j - div_ns(j, s) * s.ns;
      const float2* w = tw + s.tw_off + r;
#pragma unroll
      for (int i = 1; i < R; ++i) x[i] = twmul<DIR>(x[i], __ldg(w + (i - 1) * s.ns));
    }
    dft<R, DIR>(x);
#pragma unroll
    for (int i = 0; i < R; ++i) v[m + M * i] = x[i];
  }
}

// write the outputs of a stage to their Stockham positions in shared memory
template <int E, int R>
__device__ __forceinline__ void reg_scatter(const float2 (&v)[E], int t, int T, const Stage& s,
                                            float2* sm) {
  constexpr int M = E / R;
#pragma unroll
  for (int m = 0; m < M; ++m) {
    const int j = t + T * m;
    const int q = div_ns(j, s);
    const int base = q * s.ns * R + (j - q * s.ns);
#pragma unroll
    for (int i = 0; i < R; ++i) sm[spad(base + i * s.ns)] = v[m + M * i];
  }
}

template <int E, int DIR>
__device__ __forceinline__ void reg_stage_dispatch(float2 (&v)[E], int t, int T, const Stage& s,
                                                   const float2* __restrict__ tw) {
  switch (s.radix) {
#define PLFFT_B200_CASE(R)                                  \
  case R:                                                   \
    if constexpr (E % R == 0) reg_butterflies<E, R, DIR>(v, t, T, s, tw); \
    break;
    PLFFT_B200_RADIX_LIST(PLFFT_B200_CASE)
#undef PLFFT_B200_CASE
    default:
      break;
  }
}

template <int E>
__device__ __forceinline__ void reg_scatter_dispatch(const float2 (&v)[E], int t, int T, const Stage& s,
                                                     float2* sm) {
  switch (s.radix) {
#define PLFFT_B200_CASE(R)                                   \
  case R:                                                    \
    if constexpr (E % R == 0) reg_scatter<E, R>(v, t, T, s, sm); \
    break;
    PLFFT_B200_RADIX_LIST(PLFFT_B200_CASE)
#undef PLFFT_B200_CASE
    default:
      break;
  }
}

struct GroupSync {
  bool cta;  // true: __syncthreads, false: the group lives inside one warp
  __device__ __forceinline__ void operator()() const {
    if (cta)
      __syncthreads();
    else
      __syncwarp();
  }
};

// On entry v[q] = x[t + T*q]; on exit v[q] = X[t + T*q].
// sm: this transform's shared-memory slice (spad_len(N) complex).
template <int E, int DIR>
__device__ __forceinline__ void reg_fft(float2 (&v)[E], const FftDesc& d, int t, int T, float2* sm,
                                        const float2* __restrict__ tw, GroupSync sync) {
  reg_stage_dispatch<E, DIR>(v, t, T, d.st[0], tw);
  for (int s = 1; s < d.nstages; ++s) {
    if (s > 1) sync();  // previous exchange fully read before it is overwritten
    reg_scatter_dispatch<E>(v, t, T, d.st[s - 1], sm);
    sync();
#pragma unroll
    for (int q = 0; q < E; ++q) v[q] = sm[spad(t + T * q)];
    reg_stage_dispatch<E, DIR>(v, t, T, d.st[s], tw);
  }
}

// ===========================================================================
// Shared-memory engine (C transforms, row pitch `ld` complex each)
// ===========================================================================
template <int MAXE, int R, int DIR>
__device__ __forceinline__ void smem_stage(float2 (&x)[MAXE], float2* sm, int C, int ld, int n,
                                           const Stage& s, const float2* __restrict__ tw, int tid,
                                           int nthr) {
  constexpr int NB = MAXE / R;  // butterflies per thread
  const int nbf = n / R;
  const int total = C * nbf;
  // butterfly J = tid + b nthr as (transform c, index j), carried across b:
  // two divisions per stage instead of one per butterfly
  const int c0 = tid / nbf, j0 = tid - c0 * nbf;
  const int dq = nthr / nbf, dr = nthr - dq * nbf;
  {
    int c = c0, j = j0;
    SFor<0, NB>::run([&](auto bc) {
      constexpr int b = decltype(bc)::value;
      if (tid + b * nthr < total) {
        const float2* src = sm + c * ld;
#pragma unroll
        for (int i = 0; i < R; ++i) x[b * R + i] = src[spad(j + i * nbf)];
      }
      j += dr;
      c += dq;
      if (j >= nbf) {
        j -= nbf;
        ++c;
      }
    });
  }
  __syncthreads();
  {
    int c = c0, j = j0;
    SFor<0, NB>::run([&](auto bc) {
      constexpr int b = decltype(bc)::value;
      if (tid + b * nthr < total) {
        const int q = div_ns(j, s);
        const int r = j - q * s.ns;
        float2* xb = x + b * R;
        if (s.ns > 1) {
          const float2* w = tw + s.tw_off + r;
          if constexpr (R >= 16) {
            // a table entry every fourth factor, products with W^r between
            const float2 w1 = __ldg(w);
            float2 wi = w1;
#pragma unroll
            for (int i = 1; i < R; ++i) {
              if (i > 1) wi = (i & 3) == 1 ? __ldg(w + (i - 1) * s.ns) : cmul(wi, w1);
              xb[i] = twmul<DIR>(xb[i], wi);
            }
          } else {
#pragma unroll
            for (int i = 1; i < R; ++i) xb[i] = twmul<DIR>(xb[i], __ldg(w + (i - 1) * s.ns));
          }
        }
        dft<R, DIR>(xb);
        float2* dst = sm + c * ld;
        const int base = q * s.ns * R + r;
#pragma unroll
        for (int i = 0; i < R; ++i) dst[spad(base + i * s.ns)] = xb[i];
      }
      j += dr;
      c += dq;
      if (j >= nbf) {
        j -= nbf;
        ++c;
      }
    });
  }
  __syncthreads();
}

// In-place FFT of C transforms held in shared memory (natural order in and
// out).  Caller guarantees: for every stage, C*N/R <= (MAXE/R) * nthr.
template <int MAXE, int DIR>
__device__ __forceinline__ void smem_fft(float2* sm, int C, int ld, const FftDesc& d,
                                         const float2* __restrict__ tw, int tid, int nthr) {
  float2 x[MAXE];
  for (int s = 0; s < d.nstages; ++s) {
    switch (d.st[s].radix) {
#define PLFFT_B200_CASE(R)                                                                  \
  case R:                                                                                   \
    if constexpr (MAXE >= R) smem_stage<MAXE, R, DIR>(x, sm, C, ld, d.n, d.st[s], tw, tid, nthr); \
    break;
      PLFFT_B200_RADIX_LIST(PLFFT_B200_CASE)
#undef PLFFT_B200_CASE
      default:
        break;
    }
  }
}

}  // namespace plfft_b200
