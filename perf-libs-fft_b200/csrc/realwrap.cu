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
// four-step, Rader, Bluestein).  The reference builds the same kinds as a
// permuted R2C/C2R/C2C plus O(n) pre/post passes (src/r2r_plan.cpp:15-79,
// src/r2r_buffer_helper.hpp:231-1026); the fused single-kernel paths for the
// hot kinds live in real_fused.cu.
#include "kernels.h"
#include "stockham.cuh"

#include <algorithm>

namespace plfft_b200 {

// e^{i * sign * pi * num / den}, computed from the table of W_{4N}^m or
// directly in double for the few entries per element (FP64 is used only for
// these constants).
__device__ __forceinline__ float2 expi_pi(int64_t num, int64_t den) {
  // angle = pi * num / den, reduced modulo 2 pi in integers
  const int64_t per = 2 * den;
  int64_t m = num % per;
  if (m < 0) m += per;
  double s, c;
  sincospi(double(m) / double(den), &s, &c);
  return make_float2(float(c), float(s));
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

template <int KIND>
__device__ __forceinline__ float load_real(const RealWrapLaunch& L, int64_t b, int64_t j) {
  const float v = static_cast<const float*>(L.in)[b * L.idist + j * L.istride];
  return L.wmode_in ? v * adj_weight(L.wmode_in, j, L.n) : v;
}

template <int KIND>
__global__ void __launch_bounds__(256) realwrap_pre(const RealWrapLaunch L, int64_t m0, int64_t cnt) {
  const int64_t n = L.n, len = L.len;
  const int64_t total = cnt * len;
  for (int64_t f = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; f < total; f += int64_t(gridDim.x) * blockDim.x) {
    const int64_t bl = f / len;
    const int64_t j = f - bl * len;
    const int64_t b = m0 + bl;
    float2 z = make_float2(0.f, 0.f);
    if constexpr (KIND == RW_R2C || KIND == RW_DHT || KIND == RW_R2HC) {
      z.x = load_real<KIND>(L, b, j);
    } else if constexpr (KIND == RW_C2R) {
      const float2* X = static_cast<const float2*>(L.in) + b * L.idist;
      const int64_t h = n / 2;
      if (j <= h) {
        z = X[j * L.istride];
        if (j == 0 || (2 * j == n)) z.y = 0.f;
        if (L.wmode_in) z = cscale(z, adj_weight(L.wmode_in, j, n));
      } else {
        const float2 c = X[(n - j) * L.istride];
        z = make_float2(c.x, -c.y);
        if (L.wmode_in) z = cscale(z, adj_weight(L.wmode_in, n - j, n));
      }
    } else if constexpr (KIND == RW_HC2R) {
      const int64_t h = n / 2;
      if (j == 0) {
        z.x = load_real<KIND>(L, b, 0);
      } else if (2 * j == n) {
        z.x = load_real<KIND>(L, b, h);
      } else if (j <= h) {
        z = make_float2(load_real<KIND>(L, b, j), load_real<KIND>(L, b, n - j));
      } else {
        z = make_float2(load_real<KIND>(L, b, n - j), -load_real<KIND>(L, b, j));
      }
    } else if constexpr (KIND == RW_DCT1) {
      const int64_t src = j < n ? j : len - j;
      z.x = load_real<KIND>(L, b, src);
    } else if constexpr (KIND == RW_DCT2) {
      const int64_t src = j < n ? j : 2 * n - 1 - j;
      z.x = load_real<KIND>(L, b, src);
    } else if constexpr (KIND == RW_DST2) {
      z.x = j < n ? load_real<KIND>(L, b, j) : -load_real<KIND>(L, b, 2 * n - 1 - j);
    } else if constexpr (KIND == RW_DST1) {
      if (j >= 1 && j <= n) z.x = load_real<KIND>(L, b, j - 1);
      else if (j >= n + 2) z.x = -load_real<KIND>(L, b, len - j - 1);
    } else if constexpr (KIND == RW_DCT3) {
      if (j < n) {
        const float x = load_real<KIND>(L, b, j) * (j == 0 ? 1.f : 2.f);
        const float2 w = expi_pi(j, 2 * n);
        z = make_float2(x * w.x, x * w.y);
      }
    } else if constexpr (KIND == RW_DST3) {
      if (j >= 1 && j <= n) {
        const float x = load_real<KIND>(L, b, j - 1) * (j == n ? 1.f : 2.f);
        const float2 w = expi_pi(j, 2 * n);
        z = make_float2(x * w.x, x * w.y);
      }
    } else if constexpr (KIND == RW_DCT4 || KIND == RW_DST4) {
      if (j < n) {
        const float x = load_real<KIND>(L, b, j);
        const float2 w = expi_pi(-j, 2 * n);
        z = make_float2(x * w.x, x * w.y);
      }
    }
    L.work[bl * len + j] = z;
  }
}

template <int KIND>
__global__ void __launch_bounds__(256) realwrap_post(const RealWrapLaunch L, int64_t m0, int64_t cnt) {
  const int64_t n = L.n, len = L.len, nout = L.nout;
  const int64_t total = cnt * nout;
  const float s = L.scale;
  for (int64_t f = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; f < total; f += int64_t(gridDim.x) * blockDim.x) {
    const int64_t bl = f / nout;
    const int64_t k = f - bl * nout;
    const int64_t b = m0 + bl;
    const float2* F = L.work + bl * len;
    if constexpr (KIND == RW_R2C) {
      float2* Y = static_cast<float2*>(L.out) + b * L.odist;
      const float2 v = F[k];
      const float sw = L.wmode_out ? s * adj_weight(L.wmode_out, k, n) : s;
      Y[k * L.ostride] = make_float2(v.x * sw, v.y * sw);
    } else {
      float y = 0.f;
      if constexpr (KIND == RW_C2R || KIND == RW_HC2R || KIND == RW_DCT1 || KIND == RW_DCT3) {
        y = F[k].x;
      } else if constexpr (KIND == RW_DST3) {
        y = F[k].y;
      } else if constexpr (KIND == RW_DHT) {
        y = F[k].x - F[k].y;
      } else if constexpr (KIND == RW_R2HC) {
        y = (k <= n / 2) ? F[k].x : F[n - k].y;
      } else if constexpr (KIND == RW_DCT2) {
        const float2 w = expi_pi(-k, 2 * n);
        y = F[k].x * w.x - F[k].y * w.y;
      } else if constexpr (KIND == RW_DST2) {
        const float2 w = expi_pi(-(k + 1), 2 * n);
        const float2 v = F[k + 1];
        y = -(v.x * w.y + v.y * w.x);
      } else if constexpr (KIND == RW_DST1) {
        y = -F[k + 1].y;
      } else if constexpr (KIND == RW_DCT4 || KIND == RW_DST4) {
        const float2 w = expi_pi(-(2 * k + 1), 4 * n);
        const float2 v = F[k];
        if constexpr (KIND == RW_DCT4)
          y = 2.f * (v.x * w.x - v.y * w.y);
        else
          y = -2.f * (v.x * w.y + v.y * w.x);
      }
      const float sw = L.wmode_out ? s * adj_weight(L.wmode_out, k, n) : s;
      static_cast<float*>(L.out)[b * L.odist + k * L.ostride] = y * sw;
    }
  }
}

template <int KIND>
static cudaError_t run_pre_post(bool pre, const RealWrapLaunch& L, int64_t m0, int64_t cnt, cudaStream_t st) {
  const int64_t total = cnt * (pre ? L.len : L.nout);
  const int64_t blocks = std::min<int64_t>((total + 255) / 256, 148 * 16);
  if (pre)
    realwrap_pre<KIND><<<unsigned(std::max<int64_t>(blocks, 1)), 256, 0, st>>>(L, m0, cnt);
  else
    realwrap_post<KIND><<<unsigned(std::max<int64_t>(blocks, 1)), 256, 0, st>>>(L, m0, cnt);
  return cudaGetLastError();
}

cudaError_t launch_realwrap(bool pre, int kind, const RealWrapLaunch& L, int64_t m0, int64_t cnt, cudaStream_t st) {
  switch (kind) {
#define PLFFT_B200_RW(K) \
  case K:                \
    return run_pre_post<K>(pre, L, m0, cnt, st);
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

}  // namespace plfft_b200
