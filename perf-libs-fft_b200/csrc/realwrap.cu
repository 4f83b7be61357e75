// Real-input / real-output transforms as "pre-kernel -> C2C plan -> post-kernel".
//
// Every R2C, C2R and R2R kind is written as a complex DFT of some length L of
// a sequence built from the real input, followed by an extraction (FFTW's
// definitions, include/plfft.h:98-134, docs/plfft.md:186-212):
//
//   kind     L        built sequence z (j < L)                 output y_k
//   R2C      N        x_j                                      F_k, k <= N/2
//   C2R      N        Hermitian extension of X (Im X0, Im
//                     X_{N/2} ignored)                         Re F_k        (backward)
//   DCT-I    2(N-1)   even extension x_0..x_{N-1},x_{N-2}..x_1 Re F_k
//   DCT-II   2N       x_0..x_{N-1}, x_{N-1}..x_0              Re(e^{-i pi k/2N} F_k)
//   DCT-III  2N       c_j x_j e^{i pi j/2N}, c_0=1, c_j=2     Re F_k        (backward)
//   DCT-IV   2N       x_j e^{-i pi j/2N} (j < N)              2 Re(e^{-i pi (2k+1)/4N} F_k)
//   DST-I    2(N+1)   0, x_0..x_{N-1}, 0, -x_{N-1}..-x_0      -Im F_{k+1}
//   DST-II   2N       x_0..x_{N-1}, -x_{N-1}..-x_0            -Im(e^{-i pi (k+1)/2N} F_{k+1})
//   DST-III  2N       z_m = c_m x_{m-1} e^{i pi m/2N}, m=1..N Im F_k        (backward)
//                     (c_m = 2, c_N = 1)
//   DST-IV   2N       as DCT-IV                               -2 Im(e^{-i pi (2k+1)/4N} F_k)
//   DHT      N        x_j                                     Re F_k - Im F_k
//   R2HC     N        x_j                                     Re F_k (k <= N/2), Im F_{N-k}
//   HC2R     N        F from the half-complex layout          Re F_k        (backward)
//
// This generic path serves every length the C2C planner supports (on-chip,
// four-step, Rader, Bluestein), for FP32 data and, around the FP64 C2C
// plans, for FP64 data (the R2R kinds in double).  The reference builds the same kinds as a
// permuted R2C/C2R/C2C plus O(n) pre/post passes (src/r2r_plan.cpp:15-79,
// src/r2r_buffer_helper.hpp:231-1026); the fused single-kernel paths for the
// hot kinds live in real_fused.cu.
#include "kernels.h"
#include "stockham.cuh"

#include <algorithm>

namespace plfft_b200 {

// complex type of a real type, built component-wise so one kernel body
// serves FP32 (float2) and FP64 (double2) data
template <class R>
struct CplxOf;
template <>
struct CplxOf<float> {
  using type = float2;
};
template <>
struct CplxOf<double> {
  using type = double2;
};

template <class R>
__device__ __forceinline__ typename CplxOf<R>::type cx(R re, R im) {
  typename CplxOf<R>::type z;
  z.x = re;
  z.y = im;
  return z;
}

// e^{i pi num / den}: the angle reduced modulo 2 pi in integers, evaluated
// in double (FP32 data rounds the result once)
template <class R>
__device__ __forceinline__ typename CplxOf<R>::type expi_pi(int64_t num, int64_t den) {
  const int64_t per = 2 * den;
  int64_t m = num % per;
  if (m < 0) m += per;
  double s, c;
  sincospi(double(m) / double(den), &s, &c);
  return cx<R>(R(c), R(s));
}

// weight of element j (length n) under an AdjointWeight mode
__device__ __forceinline__ float adj_weight(int mode, int64_t j, int64_t n) {
  switch (mode) {
    case AW_HERM_HALF: return (j > 0 && 2 * j < n) ? 0.5f : 1.f;
    case AW_HERM_DOUBLE: return (j > 0 && 2 * j < n) ? 2.f : 1.f;
    case AW_FIRST_X2: return j == 0 ? 2.f : 1.f;
    case AW_FIRST_HALF: return j == 0 ? 0.5f : 1.f;
    case AW_LAST_X2: return j == n - 1 ? 2.f : 1.f;
    case AW_LAST_HALF: return j == n - 1 ? 0.5f : 1.f;
    case AW_INNER_HALF: return (j > 0 && j < n - 1) ? 0.5f : 1.f;
    case AW_INNER_X2: return (j > 0 && j < n - 1) ? 2.f : 1.f;
    case AW_HC_HALF: return (j == 0 || 2 * j == n) ? 1.f : 0.5f;
    case AW_HC_DOUBLE: return (j == 0 || 2 * j == n) ? 1.f : 2.f;
    default: return 1.f;
  }
}

template <class R>
__device__ __forceinline__ R load_real(const RealWrapLaunch& L, int64_t b, int64_t j) {
  const R v = static_cast<const R*>(L.in)[b * L.idist + j * L.istride];
  return L.wmode_in ? v * R(adj_weight(L.wmode_in, j, L.n)) : v;
}

template <class R, int KIND>
__global__ void __launch_bounds__(256) realwrap_pre(const RealWrapLaunch L, int64_t m0, int64_t cnt) {
  using C = typename CplxOf<R>::type;
  const int64_t n = L.n, len = L.len;
  const int64_t total = cnt * len;
  const bool small = total < (int64_t(1) << 31);
  C* work = static_cast<C*>(L.work);
  for (int64_t f = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; f < total; f += int64_t(gridDim.x) * blockDim.x) {
    const int64_t bl = flat_div(f, len, small);
    const int64_t j = f - bl * len;
    const int64_t b = m0 + bl;
    C z = cx<R>(0, 0);
    if constexpr (KIND == RW_R2C || KIND == RW_DHT || KIND == RW_R2HC) {
      z.x = load_real<R>(L, b, j);
    } else if constexpr (KIND == RW_C2R) {
      const C* X = static_cast<const C*>(L.in) + b * L.idist;
      const int64_t h = n / 2;
      const int64_t src = j <= h ? j : n - j;
      const C v = X[src * L.istride];
      const R w = L.wmode_in ? R(adj_weight(L.wmode_in, src, n)) : R(1);
      if (j <= h)
        z = cx<R>(v.x * w, (j == 0 || 2 * j == n) ? R(0) : v.y * w);
      else
        z = cx<R>(v.x * w, -v.y * w);
    } else if constexpr (KIND == RW_HC2R) {
      const int64_t h = n / 2;
      if (j == 0) {
        z.x = load_real<R>(L, b, 0);
      } else if (2 * j == n) {
        z.x = load_real<R>(L, b, h);
      } else if (j <= h) {
        z = cx<R>(load_real<R>(L, b, j), load_real<R>(L, b, n - j));
      } else {
        z = cx<R>(load_real<R>(L, b, n - j), -load_real<R>(L, b, j));
      }
    } else if constexpr (KIND == RW_DCT1) {
      const int64_t src = j < n ? j : len - j;
      z.x = load_real<R>(L, b, src);
    } else if constexpr (KIND == RW_DCT2) {
      const int64_t src = j < n ? j : 2 * n - 1 - j;
      z.x = load_real<R>(L, b, src);
    } else if constexpr (KIND == RW_DST2) {
      z.x = j < n ? load_real<R>(L, b, j) : -load_real<R>(L, b, 2 * n - 1 - j);
    } else if constexpr (KIND == RW_DST1) {
      if (j >= 1 && j <= n) z.x = load_real<R>(L, b, j - 1);
      else if (j >= n + 2) z.x = -load_real<R>(L, b, len - j - 1);
    } else if constexpr (KIND == RW_DCT3) {
      if (j < n) {
        const R x = load_real<R>(L, b, j) * (j == 0 ? R(1) : R(2));
        const C w = expi_pi<R>(j, 2 * n);
        z = cx<R>(x * w.x, x * w.y);
      }
    } else if constexpr (KIND == RW_DST3) {
      if (j >= 1 && j <= n) {
        const R x = load_real<R>(L, b, j - 1) * (j == n ? R(1) : R(2));
        const C w = expi_pi<R>(j, 2 * n);
        z = cx<R>(x * w.x, x * w.y);
      }
    } else if constexpr (KIND == RW_DCT4 || KIND == RW_DST4) {
      if (j < n) {
        const R x = load_real<R>(L, b, j);
        const C w = expi_pi<R>(-j, 2 * n);
        z = cx<R>(x * w.x, x * w.y);
      }
    }
    work[bl * len + j] = z;
  }
}

template <class R, int KIND>
__global__ void __launch_bounds__(256) realwrap_post(const RealWrapLaunch L, int64_t m0, int64_t cnt) {
  using C = typename CplxOf<R>::type;
  const int64_t n = L.n, len = L.len, nout = L.nout;
  const int64_t total = cnt * nout;
  const bool small = total < (int64_t(1) << 31);
  const R s = R(L.scale);
  for (int64_t f = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; f < total; f += int64_t(gridDim.x) * blockDim.x) {
    const int64_t bl = flat_div(f, nout, small);
    const int64_t k = f - bl * nout;
    const int64_t b = m0 + bl;
    const C* F = static_cast<const C*>(L.work) + bl * len;
    if constexpr (KIND == RW_R2C) {
      C* Y = static_cast<C*>(L.out) + b * L.odist;
      const C v = F[k];
      const R sw = L.wmode_out ? s * R(adj_weight(L.wmode_out, k, n)) : s;
      Y[k * L.ostride] = cx<R>(v.x * sw, v.y * sw);
    } else {
      R y = 0;
      if constexpr (KIND == RW_C2R || KIND == RW_HC2R || KIND == RW_DCT1 || KIND == RW_DCT3) {
        y = F[k].x;
      } else if constexpr (KIND == RW_DST3) {
        y = F[k].y;
      } else if constexpr (KIND == RW_DHT) {
        y = F[k].x - F[k].y;
      } else if constexpr (KIND == RW_R2HC) {
        y = (k <= n / 2) ? F[k].x : F[n - k].y;
      } else if constexpr (KIND == RW_DCT2) {
        const C w = expi_pi<R>(-k, 2 * n);
        y = F[k].x * w.x - F[k].y * w.y;
      } else if constexpr (KIND == RW_DST2) {
        const C w = expi_pi<R>(-(k + 1), 2 * n);
        const C v = F[k + 1];
        y = -(v.x * w.y + v.y * w.x);
      } else if constexpr (KIND == RW_DST1) {
        y = -F[k + 1].y;
      } else if constexpr (KIND == RW_DCT4 || KIND == RW_DST4) {
        const C w = expi_pi<R>(-(2 * k + 1), 4 * n);
        const C v = F[k];
        if constexpr (KIND == RW_DCT4)
          y = R(2) * (v.x * w.x - v.y * w.y);
        else
          y = R(-2) * (v.x * w.y + v.y * w.x);
      }
      const R sw = L.wmode_out ? s * R(adj_weight(L.wmode_out, k, n)) : s;
      static_cast<R*>(L.out)[b * L.odist + k * L.ostride] = y * sw;
    }
  }
}

template <class R, int KIND>
static cudaError_t run_pre_post(bool pre, const RealWrapLaunch& L, int64_t m0, int64_t cnt, cudaStream_t st) {
  const int64_t total = cnt * (pre ? L.len : L.nout);
  const unsigned blocks = unsigned(std::max<int64_t>(std::min<int64_t>((total + 255) / 256, 148 * 16), 1));
  if (pre)
    realwrap_pre<R, KIND><<<blocks, 256, 0, st>>>(L, m0, cnt);
  else
    realwrap_post<R, KIND><<<blocks, 256, 0, st>>>(L, m0, cnt);
  return cudaGetLastError();
}

template <class R>
static cudaError_t launch_realwrap_t(bool pre, int kind, const RealWrapLaunch& L, int64_t m0, int64_t cnt,
                                     cudaStream_t st) {
  switch (kind) {
#define PLFFT_B200_RW(K) \
  case K:                \
    return run_pre_post<R, K>(pre, L, m0, cnt, st);
    PLFFT_B200_RW(RW_R2C)
    PLFFT_B200_RW(RW_C2R)
    PLFFT_B200_RW(RW_DCT1)
    PLFFT_B200_RW(RW_DCT2)
    PLFFT_B200_RW(RW_DCT3)
    PLFFT_B200_RW(RW_DCT4)
    PLFFT_B200_RW(RW_DST1)
    PLFFT_B200_RW(RW_DST2)
    PLFFT_B200_RW(RW_DST3)
    PLFFT_B200_RW(RW_DST4)
    PLFFT_B200_RW(RW_DHT)
    PLFFT_B200_RW(RW_R2HC)
    PLFFT_B200_RW(RW_HC2R)
#undef PLFFT_B200_RW
  }
  return cudaErrorInvalidValue;
}

// Half-length R2C / C2R for even n = 2m (FP32): the n reals of a member are
// read as m complex pairs z_j = x_{2j} + i x_{2j+1}, so the complex DFT has
// length m instead of n (the split / merge of the reference's R2C / C2R
// twiddle levels, src/level_ab_t_r2c.cpp:17-120, src/level_ab_t_c2r.cpp:
// 17-99).  With W = W_n^k and Z_m = Z_0:
//   R2C, after Z = DFT_m(z):  X_k = E_k - i W O_k,  k = 0..m,
//        E_k = (Z_k + conj Z_{m-k}) / 2,  O_k = (Z_k - conj Z_{m-k}) / 2;
//   C2R, before z = IDFT_m(Z'):  Z'_k = (X_k + conj X_{m-k}) +
//        i conj(W) (X_k - conj X_{m-k}),  k < m  (Im X_0, Im X_m ignored),
//        then x_{2j} = Re z_j, x_{2j+1} = Im z_j.
// The C2C of length m reads the R2C input (writes the C2R output) in place
// of the user's buffer; these kernels are the split after it and the merge
// before it.
// (a chunk holds at most 2^23 + chunk complex values, so element indices
// within it fit 32 bits: 32-bit division instead of 64-bit)
__global__ void __launch_bounds__(256) rhalf_r2c_post(const RealHalfLaunch L, int64_t m0, int64_t cnt) {
  const uint32_t m = uint32_t(L.m);
  const uint32_t total = uint32_t(cnt) * (m + 1);
  for (uint32_t f = blockIdx.x * blockDim.x + threadIdx.x; f < total; f += gridDim.x * blockDim.x) {
    const uint32_t bl = f / (m + 1);
    const uint32_t k = f - bl * (m + 1);
    const float2* Z = L.work + size_t(bl) * m;
    const float2 zk = Z[k == m ? 0 : k];
    const float2 zm = Z[k == 0 ? 0 : m - k];
    const float2 cm = make_float2(zm.x, -zm.y);
    const float2 e = cscale(cadd(zk, cm), 0.5f);
    const float2 o = cscale(csub(zk, cm), 0.5f);
    const float2 wo = cmul(__ldg(L.tw + k), o);
    const float sw = L.wmode_out ? L.scale * adj_weight(L.wmode_out, k, 2 * m) : L.scale;
    L.out[(m0 + bl) * L.odist + int64_t(k) * L.ostride] = make_float2((e.x + wo.y) * sw, (e.y - wo.x) * sw);
  }
}

__global__ void __launch_bounds__(256) rhalf_c2r_pre(const RealHalfLaunch L, int64_t m0, int64_t cnt) {
  const uint32_t m = uint32_t(L.m);
  const uint32_t total = uint32_t(cnt) * m;
  for (uint32_t f = blockIdx.x * blockDim.x + threadIdx.x; f < total; f += gridDim.x * blockDim.x) {
    const uint32_t bl = f / m;
    const uint32_t k = f - bl * m;
    const float2* X = L.in + (m0 + bl) * L.idist;
    float2 xk = X[int64_t(k) * L.istride], xm = X[int64_t(m - k) * L.istride];
    if (L.wmode_in) {
      xk = cscale(xk, adj_weight(L.wmode_in, k, 2 * m));
      xm = cscale(xm, adj_weight(L.wmode_in, m - k, 2 * m));
    }
    if (k == 0) {  // Im X_0 and Im X_m are ignored
      xk.y = 0.f;
      xm.y = 0.f;
    }
    const float2 cm = make_float2(xm.x, -xm.y);
    const float2 a = cadd(xk, cm);
    const float2 d = csub(xk, cm);
    const float2 wd = cmulc(d, __ldg(L.tw + k));  // conj(W_n^k) d
    L.work[size_t(bl) * m + k] = cadd(a, make_float2(-wd.y, wd.x));
  }
}

cudaError_t launch_real_half(bool r2c, const RealHalfLaunch& L, int64_t m0, int64_t cnt, cudaStream_t st) {
  const int64_t total = cnt * (r2c ? L.m + 1 : L.m);
  const unsigned blocks = unsigned(std::max<int64_t>(std::min<int64_t>((total + 255) / 256, 148 * 16), 1));
  if (r2c)
    rhalf_r2c_post<<<blocks, 256, 0, st>>>(L, m0, cnt);
  else
    rhalf_c2r_pre<<<blocks, 256, 0, st>>>(L, m0, cnt);
  return cudaGetLastError();
}

cudaError_t launch_realwrap(bool pre, int kind, const RealWrapLaunch& L, int64_t m0, int64_t cnt, cudaStream_t st) {
  return L.fp64 ? launch_realwrap_t<double>(pre, kind, L, m0, cnt, st)
                : launch_realwrap_t<float>(pre, kind, L, m0, cnt, st);
}

}  // namespace plfft_b200
