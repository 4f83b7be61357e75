// Fused real-data transforms for N = 2M with M a power of two: one kernel,
// one pass over HBM.
//
// R2C  : the N reals are read as M complex values z_m = x_{2m} + i x_{2m+1};
//        Z = DFT_M(z) runs in registers; then for k = 0..M
//          X_k = E_k - i W_N^k O'_k,  E_k = (Z_k + conj Z_{M-k}) / 2,
//                                     O'_k = (Z_k - conj Z_{M-k}) / 2.
// C2R  : Z'_k = (X_k + conj X_{M-k}) + i conj(W_N^k) (X_k - conj X_{M-k})
//        (imaginary parts of X_0 and X_M ignored), z = IDFT_M(Z') gives
//        x_{2m} = Re z_m, x_{2m+1} = Im z_m.
// DCT-II: Makhoul's permutation v_j = x_{2j} (j < M), v_{N-1-j} = x_{2j+1},
//        V = DFT_N(v) by the R2C route above, then
//        y_k = 2 Re(e^{-i pi k/2N} V_k), y_{N-k} = -2 Im(e^{-i pi k/2N} V_k).
// DST-II: DST-II(x)_k = DCT-II((-1)^j x_j)_{N-1-k}.
// DCT-III (the transpose of DCT-II): with y_N = 0,
//        W_k = e^{i pi k/2N} (y_k - i y_{N-k}), k = 0..M, is a Hermitian half
//        spectrum; u = its length-N backward real DFT (the C2R route above);
//        x_{2j} = u_j, x_{2j+1} = u_{N-1-j} (Makhoul's permutation undone).
// DST-III: DST-III(y)_j = (-1)^j DCT-III(y_{N-1-k})_j.
// DCT-IV: c_p = (x_{2p} - i x_{N-1-2p}) e^{i pi p/N}, C = backward DFT_M(c),
//        S_q = e^{i pi (q + 1/4)/N} C_q: y_{2q} = 2 Re S_q, y_{N-1-2q} =
//        2 Im S_q.  DST-IV(x)_k = (-1)^k DCT-IV(x_{N-1-n})_k.
// R2HC / HC2R: the R2C / C2R routes with FFTW's half-complex order
//        (r_0 .. r_M, i_{M-1} .. i_1); DHT: H_k = Re X_k - Im X_k,
//        H_{N-k} = Re X_k + Im X_k from the R2C route.
// These are the reference's R2C / C2R twiddle levels
// (src/level_ab_t_r2c.cpp:17-120, src/level_ab_t_c2r.cpp:17-99) and its
// DCT-II / DST-II pre/post passes (src/r2r_buffer_helper.hpp:316-335,
// :455-469, :686-701, :828-854) folded into the on-chip FFT.
#pragma once
#include "kernels.h"
#include "launch_pdl.cuh"
#include "pow2_stages.cuh"
#include "ptx.cuh"

namespace plfft_b200 {

// V_k of the real length-2M input from zk = Z_k and zm = Z_{M-k}
// (Z = DFT_M(z), indices mod M) and w = W_N^k
__device__ __forceinline__ float2 split_pair(float2 zk, float2 zm, float2 w) {
  const float2 cm = make_float2(zm.x, -zm.y);
  const float2 e = cscale(cadd(zk, cm), 0.5f);
  const float2 o = cscale(csub(zk, cm), 0.5f);
  const float2 wo = cmul(w, o);
  return make_float2(e.x + wo.y, e.y - wo.x);  // e - i * wo
}

// V_k (k = 0..M) from Z held in natural order in shared memory
__device__ __forceinline__ float2 real_split(const float2* Z, int k, int m, const float2* post) {
  return split_pair(Z[k == m ? 0 : k], Z[k == 0 ? 0 : m - k], __ldg(post + k));
}

template <int M, int E, int KIND, class Sync>
__device__ __forceinline__ void finish_real(float2 (&v)[E], const RealFusedLaunch& L, float2* mine, int t,
                                            int64_t b, bool live, Sync sync) {
  using P = P2<M, E>;
  constexpr int T = P::T;
  constexpr int N = 2 * M;
  const float s = L.scale;
  if constexpr (KIND == FR_DCT4 || KIND == FR_DST4) {
    // S_q = rot_q C_q, staged as y_{2q} = 2 Re S_q, y_{N-1-2q} = +-2 Im S_q
    float* us = reinterpret_cast<float*>(mine);
    sync();  // last exchange fully read
#pragma unroll
    for (int q = 0; q < E; ++q) {
      const int m = t + T * q;
      const float2 S = cmul(__ldg(L.rot + m), v[q]);
      us[2 * m] = 2.f * S.x;
      us[N - 1 - 2 * m] = KIND == FR_DST4 ? -2.f * S.y : 2.f * S.y;
    }
    sync();
    if (!live) return;
    float* x = static_cast<float*>(L.out) + b * L.odist;
#pragma unroll
    for (int f = t; f < N; f += T) x[f] = us[f] * s;
  } else if constexpr (KIND == FR_DCT3 || KIND == FR_DST3) {
    // u_{2m} = Re z_m, u_{2m+1} = Im z_m staged as N floats, then written in
    // x order: x_{2j} = u_j, x_{2j+1} = u_{N-1-j}
    float* us = reinterpret_cast<float*>(mine);
    sync();  // last exchange fully read
#pragma unroll
    for (int q = 0; q < E; ++q) reinterpret_cast<float2*>(us)[t + T * q] = v[q];
    sync();
    if (!live) return;
    float* x = static_cast<float*>(L.out) + b * L.odist;
#pragma unroll
    for (int f = t; f < N; f += T) {
      const float u = (f & 1) ? us[N - 1 - (f >> 1)] : us[f >> 1];
      x[f] = (KIND == FR_DST3 && (f & 1)) ? -u * s : u * s;
    }
  } else if constexpr (KIND == FR_C2R || KIND == FR_HC2R) {
    if (!live) return;
    float* x = static_cast<float*>(L.out) + b * L.odist;
#pragma unroll
    for (int q = 0; q < E; ++q) {
      const int m = t + T * q;
      const float2 z = cscale(v[q], s);
      if (L.pairs_out) {
        reinterpret_cast<float2*>(x)[m] = z;
      } else {
        x[2 * m] = z.x;
        x[2 * m + 1] = z.y;
      }
    }
  } else {
    // outputs of bin k from V_k (k = 0..M)
    auto emit = [&](int k, float2 V) {
      if constexpr (KIND == FR_R2C) {
        const float sk = (L.wmode == 2 && k > 0 && k < M) ? 2.f * s : s;
        static_cast<float2*>(L.out)[b * L.odist + k] = cscale(V, sk);
      } else if constexpr (KIND == FR_R2HC || KIND == FR_DHT) {
        float* y = static_cast<float*>(L.out) + b * L.odist;
        const float re = KIND == FR_R2HC ? V.x : V.x - V.y;
        const float im = KIND == FR_R2HC ? V.y : V.x + V.y;
        y[k] = re * s;
        if (k > 0 && k < M) y[N - k] = im * s;
      } else {
        const float2 c = cmul(__ldg(L.rot + k), V);
        float* y = static_cast<float*>(L.out) + b * L.odist;
        const float yk = 2.f * c.x * s, ynk = -2.f * c.y * s;
        if constexpr (KIND == FR_DCT2) {
          y[k] = yk;
          if (k > 0 && k < M) y[N - k] = ynk;
        } else {
          y[N - 1 - k] = yk;
          if (k > 0 && k < M) y[k - 1] = ynk;
        }
      }
    };
    sync();  // last exchange fully read
#pragma unroll
    for (int q = 0; q < E; ++q) mine[t + T * q] = v[q];
    sync();
    if (!live) return;
    // k = t + T*j for j < E covers 0..M-1 (unrolled, so the table loads
    // of all j are in flight together); thread 0 also takes k = M
#pragma unroll
    for (int j = 0; j < E; ++j) emit(t + T * j, real_split(mine, t + T * j, M, L.post));
    if (t == 0) emit(M, real_split(mine, M, M, L.post));
  }
}

template <int M, int E, int KIND>
__global__ void __launch_bounds__(pow2_max_threads<E>()) real_fused_kernel(const RealFusedLaunch L) {
  griddep_wait();  // launched programmatically (launch_pdl.cuh)
  griddep_launch_dependents();
  using P = P2<M, E>;
  constexpr int T = P::T;
  constexpr int N = 2 * M;
  constexpr int PITCH = (spad_len_c(M) + 1) & ~1;
  constexpr int DIR = (KIND == FR_C2R || KIND == FR_HC2R || KIND == FR_DCT3 || KIND == FR_DST3 ||
                       KIND == FR_DCT4 || KIND == FR_DST4)
                          ? 1
                          : -1;
  extern __shared__ __align__(128) unsigned char smraw[];
  const int G = L.g;
  const int grp = threadIdx.x / T;
  const int t = threadIdx.x - grp * T;
  const int64_t b = int64_t(blockIdx.x) * G + grp;
  const bool live = b < L.howmany;
  float2* mine = reinterpret_cast<float2*>(smraw) + grp * PITCH;
  auto sync = [&]() {
    if constexpr (T <= 32)
      __syncwarp();
    else
      __syncthreads();
  };

  float2 v[E];
  if constexpr (KIND == FR_R2C || KIND == FR_R2HC || KIND == FR_DHT) {
    const float* x = static_cast<const float*>(L.in) + (live ? b * L.idist : 0);
#pragma unroll
    for (int q = 0; q < E; ++q) {
      const int m = t + T * q;
      if (!live)
        v[q] = make_float2(0.f, 0.f);
      else if (L.pairs_in)
        v[q] = reinterpret_cast<const float2*>(x)[m];
      else
        v[q] = make_float2(x[2 * m], x[2 * m + 1]);
    }
  } else if constexpr (KIND == FR_DCT4 || KIND == FR_DST4) {
    const float* xin = static_cast<const float*>(L.in) + (live ? b * L.idist : 0);
    // x_j of the (DST-IV: reversed) input
    auto X = [&](int j) { return live ? (KIND == FR_DST4 ? xin[N - 1 - j] : xin[j]) : 0.f; };
#pragma unroll
    for (int q = 0; q < E; ++q) {
      const int p = t + T * q;
      v[q] = cmul(make_float2(X(2 * p), -X(N - 1 - 2 * p)), __ldg(L.post + p));
    }
  } else if constexpr (KIND == FR_DCT3 || KIND == FR_DST3) {
    const float* y = static_cast<const float*>(L.in) + (live ? b * L.idist : 0);
    const float w0 = L.wmode == 3 ? 2.f : 1.f;
    // y_j of the (DST-III: reversed) input, y_N = 0
    auto Y = [&](int j) {
      if (!live || j >= N) return 0.f;
      const float val = KIND == FR_DST3 ? y[N - 1 - j] : y[j];
      return j == 0 ? w0 * val : val;
    };
    // W_k = conj(rot_k) (y_k - i y_{N-k})
    auto Wk = [&](int k) { return cmulc(make_float2(Y(k), -Y(N - k)), __ldg(L.rot + k)); };
#pragma unroll
    for (int q = 0; q < E; ++q) {
      const int k = t + T * q;
      float2 xk = Wk(k), xm = Wk(M - k);
      const bool k0 = k == 0;  // imaginary parts of W_0 and W_M ignored
      xk.y = k0 ? 0.f : xk.y;
      xm.y = k0 ? 0.f : xm.y;
      const float2 cm = make_float2(xm.x, -xm.y);
      const float2 a = cadd(xk, cm);
      const float2 d = csub(xk, cm);
      const float2 wd = cmulc(d, __ldg(L.post + k));  // conj(W_N^k) * d
      v[q] = cadd(a, make_float2(-wd.y, wd.x));       // a + i * wd
    }
  } else if constexpr (KIND == FR_HC2R) {
    const float* h = static_cast<const float*>(L.in) + (live ? b * L.idist : 0);
    // X_j = (r_j, i_j) read from the half-complex order, i_0 = i_M = 0
    auto Xj = [&](int j) {
      const bool inner = j > 0 && j < M;
      return live ? make_float2(h[j], inner ? h[inner ? N - j : 0] : 0.f) : make_float2(0.f, 0.f);
    };
#pragma unroll
    for (int q = 0; q < E; ++q) {
      const int k = t + T * q;
      const float2 xk = Xj(k), xm = Xj(M - k);
      const float2 cm = make_float2(xm.x, -xm.y);
      const float2 a = cadd(xk, cm);
      const float2 d = csub(xk, cm);
      const float2 wd = cmulc(d, __ldg(L.post + k));  // conj(W_N^k) * d
      v[q] = cadd(a, make_float2(-wd.y, wd.x));       // a + i * wd
    }
  } else if constexpr (KIND == FR_C2R) {
    const float2* X = static_cast<const float2*>(L.in) + (live ? b * L.idist : 0);
    const float hw = L.wmode == 1 ? 0.5f : 1.f;
#pragma unroll
    for (int q = 0; q < E; ++q) {
      const int k = t + T * q;
      if (!live) {
        v[q] = make_float2(0.f, 0.f);
        continue;
      }
      float2 xk = X[k], xm = X[M - k];
      // k = 0: imaginary parts of X_0 and X_M ignored; adjoint weights halve
      // bins 0 < k < M (both k and M - k here); selects, not branches, so
      // the loads of every q stay in flight together
      const bool k0 = k == 0;
      const float w = k0 ? 1.f : hw;
      xk = make_float2(xk.x * w, k0 ? 0.f : xk.y * w);
      xm = make_float2(xm.x * w, k0 ? 0.f : xm.y * w);
      const float2 cm = make_float2(xm.x, -xm.y);
      const float2 a = cadd(xk, cm);
      const float2 d = csub(xk, cm);
      const float2 wd = cmulc(d, __ldg(L.post + k));  // conj(W_N^k) * d
      v[q] = cadd(a, make_float2(-wd.y, wd.x));       // a + i * wd
    }
  } else if (T <= 32 && L.quads_in) {  // T is a compile-time constant
    // DCT-II / DST-II from aligned float4 loads, no staging: x_{4m..4m+3}
    // (m < M/2) holds z_m = (x_{4m}, x_{4m+2}) and z_{M-1-m} = (x_{4m+3},
    // x_{4m+1}) of the Makhoul-permuted pairs.  For m = t + T q, z_{M-1-m}
    // is element E-1-q of lane T-1-t (t XOR (T-1), same warp as T <= 32),
    // so the two lanes swap those halves with one shuffle per component.
    const float4* x4 = reinterpret_cast<const float4*>(static_cast<const float*>(L.in) + (live ? b * L.idist : 0));
#pragma unroll
    for (int q = 0; q < E / 2; ++q) {
      float4 a = live ? x4[t + T * q] : make_float4(0.f, 0.f, 0.f, 0.f);
      if constexpr (KIND == FR_DST2) {
        a.y = -a.y;
        a.w = -a.w;
      }
      v[q] = make_float2(a.x, a.z);
      v[E - 1 - q] = make_float2(__shfl_xor_sync(0xffffffffu, a.w, T - 1), __shfl_xor_sync(0xffffffffu, a.y, T - 1));
    }
  } else {
    // DCT-II / DST-II: stage the N reals in the slot, then gather the
    // Makhoul-permuted pairs
    float* xs = reinterpret_cast<float*>(mine);
    const float* x = static_cast<const float*>(L.in) + (live ? b * L.idist : 0);
#pragma unroll
    for (int f = t; f < N; f += T) {
      float val = live ? x[f] : 0.f;
      if constexpr (KIND == FR_DST2) val = (f & 1) ? -val : val;
      xs[f] = val;
    }
    sync();
    auto perm = [&](int j) { return j < M ? xs[2 * j] : xs[2 * (N - 1 - j) + 1]; };
#pragma unroll
    for (int q = 0; q < E; ++q) {
      const int m = t + T * q;
      v[q] = make_float2(perm(2 * m), perm(2 * m + 1));
    }
  }

  // stage twiddles: the lookup-every-fourth recurrence for E = 32 (R2C+C2R
  // N=4096: 3.09 against 2.98 TB/s), table entries for E = 16 (DCT-II
  // N=1024: 1.82 against 1.49 TB/s with the recurrence)
  constexpr int RMIN = E >= 32 ? 16 : 64;
  st_bfly<T, E, P::radix(0), 1, 0, DIR, false, RMIN>(v, t, L.tw);
  Stages<N / 2, E, DIR, 1, false, RMIN>::run(v, t, mine, L.tw, sync);
  finish_real<M, E, KIND>(v, L, mine, t, b, live, sync);
}

template <int M, int E, int KIND>
cudaError_t run_real_fused(const RealFusedLaunch& L, cudaStream_t st) {
  constexpr int T = M / E;
  constexpr int PITCH = (spad_len_c(M) + 1) & ~1;
  const int smem = L.g * PITCH * int(sizeof(float2));
  {
    const cudaError_t e = ensure_dynamic_smem(reinterpret_cast<const void*>(real_fused_kernel<M, E, KIND>), smem);
    if (e != cudaSuccess) return e;
  }
  const int64_t blocks = (L.howmany + L.g - 1) / L.g;
  return launch_pdl(real_fused_kernel<M, E, KIND>, dim3(unsigned(blocks)), dim3(T * L.g), size_t(smem), st, L);
}

// every length of one kind (m = 512 has a 16- and a 32-element form)
template <int KIND>
cudaError_t launch_real_fused_kind(int m, const RealFusedLaunch& L, cudaStream_t st) {
  switch (m) {
    case 64: return run_real_fused<64, 16, KIND>(L, st);
    case 128: return run_real_fused<128, 16, KIND>(L, st);
    case 256: return run_real_fused<256, 16, KIND>(L, st);
    case 512: return L.e == 32 ? run_real_fused<512, 32, KIND>(L, st) : run_real_fused<512, 16, KIND>(L, st);
    case 1024: return run_real_fused<1024, 32, KIND>(L, st);
    case 2048: return run_real_fused<2048, 32, KIND>(L, st);
    case 4096: return run_real_fused<4096, 16, KIND>(L, st);
    case 8192: return run_real_fused<8192, 32, KIND>(L, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace plfft_b200
