// Radix-R DFT codelets for FP32 complex data held in registers.
//
// These replace the base "codelet" kernels of the reference
// (src/providers/jit/wfta_nfact.cpp:22-171 generates the radix-2..20 DAGs
// that the AArch64 kernels evaluate; src/kernel_function_pointers.hpp:12-40
// gives their call signatures).  On the GPU a codelet is an inline device
// function over an array of R complex registers; the surrounding Stockham
// engine (stockham.cuh) supplies the data movement that the reference's
// howmany/stride loops did.
//
// Direction convention: DIR = -1 forward (exp(-2 pi i jk/R)), +1 backward.
// Constants are evaluated at compile time in double precision
// (constexpr Taylor series, own implementation) and rounded once to float.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>
#include <utility>

namespace plfft_b200 {

// ---------------------------------------------------------------------------
// complex helpers
// ---------------------------------------------------------------------------
struct cf {
  float x, y;
};

// Complex arithmetic on float2.  sm_100 executes two FP32 lanes per
// instruction (FADD2/FMUL2/FFMA2), so re and im share one instruction.
// a - b is formed as fma(b, -1, a): exact negation, one rounding, the same
// result as a subtraction.
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) {
  return __ffma2_rn(b, make_float2(-1.f, -1.f), a);
}
// a * b = (a.x b.x - a.y b.y, a.x b.y + a.y b.x)
//       = a.x * (b.x, b.y) + a.y * (-b.y, b.x)
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  const float2 t = __fmul2_rn(make_float2(a.x, a.x), b);
  return __ffma2_rn(make_float2(a.y, a.y), make_float2(-b.y, b.x), t);
}
// a * conj(b) = a.x * (b.x, -b.y) + a.y * (b.y, b.x)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
  const float2 t = __fmul2_rn(make_float2(a.x, a.x), make_float2(b.x, -b.y));
  return __ffma2_rn(make_float2(a.y, a.y), make_float2(b.y, b.x), t);
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return __fmul2_rn(a, make_float2(s, s)); }
// multiply by (s * i) where s = +1 or -1 (compile time)
template <int S>
__device__ __forceinline__ float2 cmul_i(float2 a) {
  return S > 0 ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}
// twiddle multiply: DIR=-1 uses the table value w, DIR=+1 uses conj(w)
template <int DIR>
__device__ __forceinline__ float2 twmul(float2 a, float2 w) {
  return DIR < 0 ? cmul(a, w) : cmulc(a, w);
}

// ---------------------------------------------------------------------------
// compile-time trigonometry (double precision)
// ---------------------------------------------------------------------------
namespace ce {
constexpr double kPi = 3.14159265358979323846264338327950288;
constexpr double sin_poly(double x) {
  // Taylor series on |x| <= pi/4, 14 terms: error far below 1 ulp of double
  double x2 = x * x, term = x, sum = x;
  for (int k = 1; k < 14; ++k) {
    term *= -x2 / double((2 * k) * (2 * k + 1));
    sum += term;
  }
  return sum;
}
constexpr double cos_poly(double x) {
  double x2 = x * x, term = 1.0, sum = 1.0;
  for (int k = 1; k < 14; ++k) {
    term *= -x2 / double((2 * k - 1) * (2 * k));
    sum += term;
  }
  return sum;
}
// cos and sin of 2*pi*k/n, exact at multiples of 1/8 turn
struct cs {
  double c, s;
};
constexpr cs unit_root(long long k, long long n) {
  k %= n;
  if (k < 0) k += n;
  // octant reduction in integer arithmetic: angle = (8k/n) * pi/4
  long long k8 = 8 * k;
  long long oct = k8 / n;          // 0..7
  long long rem = k8 - oct * n;    // angle within octant = rem/n * pi/4
  double r = double(rem) / double(n) * (kPi / 4.0);
  // reduce into [-pi/8, pi/8] style: use octant pairs
  double c0 = 0.0, s0 = 0.0;
  if (oct % 2 == 0) {
    c0 = cos_poly(r);
    s0 = sin_poly(r);
  } else {
    // angle = (oct+1)*pi/4 - (pi/4 - r)
    double r2 = kPi / 4.0 - r;
    c0 = cos_poly(r2);
    s0 = -sin_poly(r2);
    oct += 1;
  }
  // now angle = oct*pi/4 + t with cos t = c0, sin t = s0 (oct even)
  long long q = (oct / 2) % 4;
  double c = c0, s = s0;
  if (q == 1) { c = -s0; s = c0; }
  if (q == 2) { c = -c0; s = -s0; }
  if (q == 3) { c = s0; s = -c0; }
  return {c, s};
}
}  // namespace ce

// W_n^k = exp(DIR * 2 pi i k / n) as a float2, evaluated at compile time
template <int DIR, int N, int K>
struct Root {
  static constexpr ce::cs v = ce::unit_root(K, N);
  static constexpr float re = float(v.c);
  static constexpr float im = float(DIR * v.s);
};
template <int N, int K>
struct RootCos {
  static constexpr float v = float(ce::unit_root(K, N).c);
};
template <int N, int K>
struct RootSin {
  static constexpr float v = float(ce::unit_root(K, N).s);
};

// ---------------------------------------------------------------------------
// static loop helper
// ---------------------------------------------------------------------------
template <int I, int END>
struct SFor {
  template <class F>
  __device__ __forceinline__ static void run(F&& f) {
    if constexpr (I < END) {
      f(std::integral_constant<int, I>{});
      SFor<I + 1, END>::run(f);
    }
  }
};

// ---------------------------------------------------------------------------
// prime-radix codelet via symmetric pairs, R odd prime
//   X[m] = A_m + s*i*B_m,  X[R-m] = A_m - s*i*B_m
//   A_m = x0 + sum_k (x_k + x_{R-k}) cos(2 pi mk/R)
//   B_m =      sum_k (x_k - x_{R-k}) sin(2 pi mk/R)
// ---------------------------------------------------------------------------
template <int R, int DIR>
__device__ __forceinline__ void dft_odd(float2* v) {
  constexpr int H = (R - 1) / 2;
  float2 a[H + 1], b[H + 1];
  float2 x0 = v[0];
  float2 sum = x0;
#pragma unroll
  for (int k = 1; k <= H; ++k) {
    a[k] = cadd(v[k], v[R - k]);
    b[k] = csub(v[k], v[R - k]);
    sum = cadd(sum, a[k]);
  }
  float2 out[R];
  out[0] = sum;
  SFor<1, H + 1>::run([&](auto mc) {
    constexpr int m = decltype(mc)::value;
    float2 A = x0, B = make_float2(0.f, 0.f);
    SFor<1, H + 1>::run([&](auto kc) {
      constexpr int k = decltype(kc)::value;
      constexpr float c = RootCos<R, (m * k) % R>::v;
      constexpr float s = RootSin<R, (m * k) % R>::v;
      A = __ffma2_rn(a[k], make_float2(c, c), A);
      B = __ffma2_rn(b[k], make_float2(s, s), B);
    });
    // s*i*B with s = DIR
    float2 iB = cmul_i<DIR>(B);
    out[m] = cadd(A, iB);
    out[R - m] = csub(A, iB);
  });
#pragma unroll
  for (int k = 0; k < R; ++k) v[k] = out[k];
}

template <int R, int DIR>
__device__ __forceinline__ void dft(float2* v);

template <int DIR>
__device__ __forceinline__ void dft2(float2* v) {
  float2 a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <int DIR>
__device__ __forceinline__ void dft4(float2* v) {
  float2 t0 = cadd(v[0], v[2]);
  float2 t1 = csub(v[0], v[2]);
  float2 t2 = cadd(v[1], v[3]);
  float2 t3 = cmul_i<DIR>(csub(v[1], v[3]));
  v[0] = cadd(t0, t2);
  v[2] = csub(t0, t2);
  v[1] = cadd(t1, t3);
  v[3] = csub(t1, t3);
}

// composite radix R = R1 * R2 in registers:
//   n = R2*n1 + n2, k = k1 + R1*k2
//   A[n2][k1] = DFT_R1 over n1 of x[R2 n1 + n2]; A *= W_R^{n2 k1};
//   X[k1 + R1 k2] = DFT_R2 over n2 of A[n2][k1]
template <int R1, int R2, int DIR>
__device__ __forceinline__ void dft_composite(float2* v) {
  constexpr int R = R1 * R2;
  float2 a[R];
  SFor<0, R2>::run([&](auto n2c) {
    constexpr int n2 = decltype(n2c)::value;
    float2 t[R1];
#pragma unroll
    for (int n1 = 0; n1 < R1; ++n1) t[n1] = v[R2 * n1 + n2];
    dft<R1, DIR>(t);
    SFor<0, R1>::run([&](auto k1c) {
      constexpr int k1 = decltype(k1c)::value;
      constexpr int e = (n2 * k1) % R;
      if constexpr (e == 0) {
        a[n2 * R1 + k1] = t[k1];
      } else if constexpr (4 * e == R) {
        a[n2 * R1 + k1] = cmul_i<DIR>(t[k1]);
      } else if constexpr (4 * e == 3 * R) {
        a[n2 * R1 + k1] = cmul_i<-DIR>(t[k1]);
      } else if constexpr (2 * e == R) {
        a[n2 * R1 + k1] = make_float2(-t[k1].x, -t[k1].y);
      } else {
        constexpr float wr = Root<DIR, R, e>::re;
        constexpr float wi = Root<DIR, R, e>::im;
        a[n2 * R1 + k1] = cmul(t[k1], make_float2(wr, wi));
      }
    });
  });
  SFor<0, R1>::run([&](auto k1c) {
    constexpr int k1 = decltype(k1c)::value;
    float2 t[R2];
#pragma unroll
    for (int n2 = 0; n2 < R2; ++n2) t[n2] = a[n2 * R1 + k1];
    dft<R2, DIR>(t);
#pragma unroll
    for (int k2 = 0; k2 < R2; ++k2) v[k1 + R1 * k2] = t[k2];
  });
}

template <int R, int DIR>
__device__ __forceinline__ void dft(float2* v) {
  if constexpr (R == 1) {
  } else if constexpr (R == 2) {
    dft2<DIR>(v);
  } else if constexpr (R == 4) {
    dft4<DIR>(v);
  } else if constexpr (R == 3 || R == 5 || R == 7 || R == 11 || R == 13) {
    dft_odd<R, DIR>(v);
  } else if constexpr (R == 8) {
    dft_composite<2, 4, DIR>(v);
  } else if constexpr (R == 16) {
    dft_composite<4, 4, DIR>(v);
  } else if constexpr (R == 32) {
    dft_composite<4, 8, DIR>(v);
  } else if constexpr (R == 64) {
    dft_composite<8, 8, DIR>(v);
  } else if constexpr (R == 6) {
    dft_composite<2, 3, DIR>(v);
  } else if constexpr (R == 9) {
    dft_composite<3, 3, DIR>(v);
  } else if constexpr (R == 10) {
    dft_composite<2, 5, DIR>(v);
  } else if constexpr (R == 12) {
    dft_composite<4, 3, DIR>(v);
  } else if constexpr (R == 14) {
    dft_composite<2, 7, DIR>(v);
  } else if constexpr (R == 15) {
    dft_composite<3, 5, DIR>(v);
  } else {
    static_assert(R == 2, "unsupported radix");
  }
}

// Radices the engines can dispatch at run time.
#define PLFFT_B200_RADIX_LIST(X) X(2) X(3) X(4) X(5) X(7) X(8) X(11) X(13) X(16) X(32)

}  // namespace plfft_b200
