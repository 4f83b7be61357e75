// Compile-time Stockham stage list for power-of-two transforms held in
// registers: N = R0 * E^(S-1), T = N/E threads per transform.  Shared by
// the C2C kernels (c2c_pow2.cu) and the fused real kernels (real_fused.cu).
#pragma once
#include "stockham.cuh"

namespace plfft_b200 {

template <int N, int E>
struct P2 {
  static constexpr int count_e(int m) { return (m % E == 0 && m > 1) ? 1 + count_e(m / E) : 0; }
  static constexpr int pow_e(int k) { return k == 0 ? 1 : E * pow_e(k - 1); }
  static constexpr int KE = count_e(N);           // number of full radix-E stages
  static constexpr int REST = N / pow_e(KE);      // leftover factor (1 or < E)
  static constexpr int S = KE + (REST > 1 ? 1 : 0);
  static constexpr int R0 = REST > 1 ? REST : E;
  static constexpr int T = N / E;
  static constexpr int radix(int s) { return s == 0 ? R0 : E; }
  static constexpr int ns(int s) { return s == 0 ? 1 : R0 * pow_e(s - 1); }
  static constexpr int twoff(int s) { return s <= 1 ? 0 : twoff(s - 1) + (E - 1) * ns(s - 1); }
};

// TWS: the twiddle table lives in shared memory (plain loads) instead of
// global memory (read-only cache loads)
// RMIN: smallest radix whose twiddles use the lookup-every-fourth recurrence
template <int T, int E, int R, int NS, int TWOFF, int DIR, bool TWS = false, int RMIN = 16>
__device__ __forceinline__ void st_bfly(float2 (&v)[E], int t, const float2* __restrict__ tw) {
  constexpr int M = E / R;
#pragma unroll
  for (int m = 0; m < M; ++m) {
    float2 x[R];
#pragma unroll
    for (int i = 0; i < R; ++i) x[i] = v[m + M * i];
    if constexpr (NS > 1) {
      const int j = t + T * m;
      const int r = j & (NS - 1);
      const float2* w = tw + TWOFF + r;
      // W^{r i} for i = 1..R-1: for R >= 16 a table entry every fourth i
      // and products with W^r in between (at most three extra roundings,
      // a quarter of the loads); small radices load every entry
      auto load = [&](int i) {
        if constexpr (TWS)
          return w[(i - 1) * NS];
        else
          return __ldg(w + (i - 1) * NS);
      };
      if constexpr (R >= RMIN) {
        const float2 w1 = load(1);
        float2 wi = w1;
#pragma unroll
        for (int i = 1; i < R; ++i) {
          if (i > 1) wi = (i & 3) == 1 ? load(i) : cmul(wi, w1);
          x[i] = twmul<DIR>(x[i], wi);
        }
      } else {
#pragma unroll
        for (int i = 1; i < R; ++i) x[i] = twmul<DIR>(x[i], load(i));
      }
    }
    dft<R, DIR>(x);
#pragma unroll
    for (int i = 0; i < R; ++i) v[m + M * i] = x[i];
  }
}

// Exchange padding: one spare complex every 2^PS.  A stage's scatter
// writes, for a fixed output i, the 16 threads of a half-warp to addresses
// R (j / NS) NS + j mod NS + i NS: with one spare every 16 complex, radix
// <= 16 rows land on 16 distinct 8-byte bank pairs, but radix-32 rows (a
// stride of 34) collide two ways; one spare every 32 (a stride of 33)
// separates them.  Each exchange picks its own padding (the gather that
// follows uses the same), sized within spad_len().
template <int R>
constexpr int exchange_pad_shift() { return R >= 32 ? 5 : 4; }
template <int PS>
__device__ __forceinline__ int xpad(int p) { return p + (p >> PS); }

template <int T, int E, int R, int NS>
__device__ __forceinline__ void st_scatter(const float2 (&v)[E], int t, float2* sm) {
  constexpr int M = E / R;
  constexpr int PS = exchange_pad_shift<R>();
#pragma unroll
  for (int m = 0; m < M; ++m) {
    const int j = t + T * m;
    const int base = (j & ~(NS - 1)) * R + (j & (NS - 1));
#pragma unroll
    for (int i = 0; i < R; ++i) sm[xpad<PS>(base + i * NS)] = v[m + M * i];
  }
}

template <int N, int E, int DIR, int S, bool TWS = false, int RMIN = 16>
struct Stages {
  using P = P2<N, E>;
  template <class Sync>
  __device__ __forceinline__ static void run(float2 (&v)[E], int t, float2* xb, const float2* tw, Sync sync) {
    if constexpr (S < P::S) {
      sync();  // the buffer's previous contents are fully read
      st_scatter<P::T, E, P::radix(S - 1), P::ns(S - 1)>(v, t, xb);
      sync();
      constexpr int PS = exchange_pad_shift<P::radix(S - 1)>();
#pragma unroll
      for (int q = 0; q < E; ++q) v[q] = xb[xpad<PS>(t + P::T * q)];
      st_bfly<P::T, E, P::radix(S), P::ns(S), P::twoff(S), DIR, TWS, RMIN>(v, t, tw);
      Stages<N, E, DIR, S + 1, TWS, RMIN>::run(v, t, xb, tw, sync);
    }
  }
};

template <int E>
constexpr int pow2_max_threads() { return E <= 16 ? 512 : 256; }
// minimum resident blocks for __launch_bounds__: caps E=32 kernels at 128
// registers (they fit without spilling), which doubles the warps per SM
template <int E>
constexpr int pow2_min_blocks() { return E <= 16 ? 1 : 2; }

}  // namespace plfft_b200
