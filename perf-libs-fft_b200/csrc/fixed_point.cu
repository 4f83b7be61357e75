// Fixed-point C2C, Q0.15 (B = 16) and Q0.7 (B = 8), power-of-two n <= 4096,
// bit-exact to the reference's NEON fixed-point path.
//
// Arithmetic (reference src/providers/jit/print_algo.cpp:1228-1230,
// src/providers/jit/emit.hpp:150-175 and :370-425, constant lowering
// print_algo.cpp:2150-2290): codelet inputs are pre-scaled by a rounding
// shift right by log2(radix); additions saturate to B bits; a real-constant
// multiply is (a k + 2^(B-2)) >> (B-1) (sqrdmulh for Q0.15, smull + sqrshrn
// #7 for Q0.7); a twiddle product is two B x B products accumulated in a
// 2B-bit lane and narrowed by one rounding, saturating shift by B - 1.  The
// codelets are radix 2, 4, 8 and the fixed-point split-radix 16
// (src/providers/jit/split_radix_z16.cpp, src/providers/jit/wfta_nfact.cpp:
// 89-97); a backward codelet of length r yields the forward codelet's
// output r-k at index k.  Decomposition = the reference's ESTIMATE plan
// (planner/planner.cpp:51-175 with base kernels {2, 4, 8, 16}):
//   n <= 16     one codelet;
//   n = 16 m    cooley_tukey_ab(16) (planner/strategies/cooley_tukey.hpp:
//               82-143, 622-680): length-m codelets down the 16 columns
//               x[c + 16 q], then per row j a 16-point codelet whose inputs
//               i >= 1 are multiplied by the twiddle of W_n^{dir i j},
//               output y[j + m k];
//   n = 256 m'  the length-16 m' sub-transforms of that plan are
//               cooley_tukey_ac(16) (cooley_tukey.hpp:331-385, 682-748):
//               length-m' codelets down the 256 columns x[c + 256 q], then
//               for column t < 16 and row i0 < m' a 16-point codelet over
//               b1[256 i0 + t + 16 i] (rows i0 >= 1 twiddled by
//               W_{16 m'}^{dir i i0}) into b0[16 i0 + t + 16 m' k], then the
//               twiddled rows of the n = 16 m case over b0.
// Twiddles are the reference's premultiplied pairs (src/generate_twiddles.hpp:
// 72-132), passed as short4 (c, s, cvt(-s), c).
//
// Saturation: every codelet input is pre-shifted by log2(r), so an interval
// analysis of each codelet (tests/test_q15.py::test_q15_codelet_
// intermediates_never_saturate and ::test_q7_codelet_intermediates_never_
// saturate) shows that only the final output additions can leave B bits and
// that no MAC lane wraps; intermediates therefore use plain integer
// arithmetic (identical results) and outputs saturate when packed.
//
// GPU mapping: members are staged in shared memory at padded position
// k + k/16 (a column and a row are both read without bank conflicts).
// n = 16 m: a CTA takes G members, 16 threads per member run the column
// codelets in place, then one thread per row runs the twiddled 16-point
// codelet and stores its outputs.  n = 256 m': one member per CTA of 256
// threads: one column codelet per thread, one (column, row) task of the
// inner level per thread, one outer row per thread.
#include <stdint.h>

#include <type_traits>

#include "kernels.h"
#include "launch_pdl.cuh"
#include "ptx.cuh"

namespace plfft_b200 {

struct qc {
  int re, im;
};

// lane format: storage word of one complex element and the Q0.(B-1) constants
template <int B>
struct Fx;
template <>
struct Fx<16> {
  using W = int;  // int16 (re, im), re in the low half
  static constexpr int LO = -32768, HI = 32767;
  static constexpr int C8 = 23170, C16 = 30273, S16 = 12539;  // trunc(2^15 cos/sin)
};
template <>
struct Fx<8> {
  using W = short;  // int8 (re, im), re in the low byte
  static constexpr int LO = -128, HI = 127;
  static constexpr int C8 = 90, C16 = 118, S16 = 48;  // trunc(2^7 cos/sin)
};

__device__ __forceinline__ int rshr(int v, int s) { return (v + (1 << (s - 1))) >> s; }

template <int B>
struct Ar {
  // multiply by a real constant k: never saturates for the operands that
  // reach it (interval analysis)
  template <int K>
  __device__ __forceinline__ static int rdm(int a) {
    static_assert(K >= Fx<B>::LO && K <= Fx<B>::HI, "constant out of range");
    return (a * K + (1 << (B - 2))) >> (B - 1);
  }
  __device__ __forceinline__ static int mac2(int a, int ka, int b, int kb) {
    return (a * ka + b * kb + (1 << (B - 2))) >> (B - 1);
  }
  __device__ __forceinline__ static qc add(qc a, qc b) { return {a.re + b.re, a.im + b.im}; }
  __device__ __forceinline__ static qc sub(qc a, qc b) { return {a.re - b.re, a.im - b.im}; }
  // -1 times a value in range is exact
  __device__ __forceinline__ static qc mul_pi(qc z) { return {-z.im, rdm<Fx<B>::HI>(z.re)}; }
  __device__ __forceinline__ static qc mul_mi(qc z) { return {rdm<Fx<B>::HI>(z.im), -z.re}; }
  __device__ __forceinline__ static qc mul_w8(qc z) {
    constexpr int C = Fx<B>::C8;
    return {mac2(z.re, C, rdm<C>(z.im), Fx<B>::HI), mac2(z.im, C, rdm<C>(z.re), Fx<B>::LO)};
  }
  __device__ __forceinline__ static qc mul_w8_3(qc z) {
    constexpr int C = -Fx<B>::C8;
    return {mac2(z.re, C, rdm<C>(z.im), Fx<B>::LO), mac2(z.im, C, rdm<C>(z.re), Fx<B>::HI)};
  }
  __device__ __forceinline__ static qc mul_w(qc z, int wr, int wi) {
    return {mac2(z.re, wr, z.im, -wi), mac2(z.im, wr, z.re, wi)};
  }
  // twiddle (c, s, cvt(-s), c): one rounding per component
  __device__ __forceinline__ static qc twiddle(qc s, short4 w) {
    return {mac2(s.re, w.x, s.im, w.z), mac2(s.re, w.y, s.im, w.w)};
  }
};

// ---- codelets on pre-scaled inputs, outputs in forward order ----
template <int B>
__device__ __forceinline__ void q_dft2(const qc* a, qc* y) {
  using A = Ar<B>;
  y[0] = A::add(a[0], a[1]);
  y[1] = A::sub(a[0], a[1]);
}

template <int B>
__device__ __forceinline__ void q_dft4(const qc* a, qc* y) {
  using A = Ar<B>;
  const qc s02 = A::add(a[0], a[2]), s13 = A::add(a[1], a[3]);
  const qc d02 = A::sub(a[0], a[2]), j13 = A::mul_pi(A::sub(a[1], a[3]));
  y[0] = A::add(s02, s13);
  y[2] = A::sub(s02, s13);
  y[1] = A::sub(d02, j13);
  y[3] = A::add(d02, j13);
}

template <int B>
__device__ __forceinline__ void q_dft8(const qc* a, qc* y) {
  using A = Ar<B>;
  constexpr int C8 = Fx<B>::C8, HI = Fx<B>::HI, LO = Fx<B>::LO;
  qc p[4], m[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    p[k] = A::add(a[k], a[k + 4]);
    m[k] = A::sub(a[k], a[k + 4]);
  }
  const qc e0 = A::add(p[0], p[2]), e1 = A::add(p[1], p[3]);
  y[0] = A::add(e0, e1);
  y[4] = A::sub(e0, e1);
  const qc d = A::sub(p[0], p[2]), jd = A::mul_pi(A::sub(p[1], p[3]));
  y[2] = A::sub(d, jd);
  y[6] = A::add(d, jd);
  const qc z = A::add(m[1], m[3]), w = A::sub(m[1], m[3]);
  const qc rd = {A::template rdm<C8>(w.re), A::template rdm<C8>(w.im)};
  const qc x = {A::mac2(m[2].im, LO, z.im, -C8), A::mac2(m[2].re, HI, z.re, C8)};
  const qc x2 = {A::mac2(m[2].im, LO, z.im, C8), A::mac2(m[2].re, HI, z.re, -C8)};
  const qc u = A::add(m[0], rd), v = A::sub(m[0], rd);
  y[1] = A::sub(u, x);
  y[7] = A::add(u, x);
  y[3] = A::add(v, x2);
  y[5] = A::sub(v, x2);
}

template <int B>
__device__ __forceinline__ void q_dft16(const qc* a, qc* y) {
  using A = Ar<B>;
  constexpr int C16 = Fx<B>::C16, S16 = Fx<B>::S16;
  qc p[8], m[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    p[k] = A::add(a[k], a[k + 8]);
    m[k] = A::sub(a[k], a[k + 8]);
  }
  const qc s04 = A::add(p[0], p[4]), s26 = A::add(p[2], p[6]);
  const qc s15 = A::add(p[1], p[5]), s37 = A::add(p[3], p[7]);
  const qc e0 = A::add(s04, s26), e1 = A::add(s15, s37);
  y[0] = A::add(e0, e1);
  y[8] = A::sub(e0, e1);
  const qc Aq = A::sub(s04, s26), jB = A::mul_pi(A::sub(s15, s37));
  y[4] = A::sub(Aq, jB);
  y[12] = A::add(Aq, jB);
  const qc C = A::sub(p[0], p[4]), jD = A::mul_pi(A::sub(p[2], p[6]));
  const qc kE = A::mul_w8(A::sub(p[1], p[5])), kF = A::mul_w8_3(A::sub(p[3], p[7]));
  const qc g1 = A::sub(C, jD), g2 = A::add(C, jD);
  const qc h = A::add(kE, kF), h2 = A::mul_mi(A::sub(kF, kE));
  y[2] = A::add(g1, h);
  y[10] = A::sub(g1, h);
  y[6] = A::sub(g2, h2);
  y[14] = A::add(g2, h2);
  const qc j4 = A::mul_pi(m[4]);
  const qc q = A::sub(m[0], j4), q2 = A::add(m[0], j4);
  const qc k2 = A::mul_w8(m[2]), k6 = A::mul_w8_3(m[6]);
  const qc r = A::add(k2, k6), r2 = A::mul_mi(A::sub(k6, k2));
  const qc j5 = A::mul_pi(m[5]), j7 = A::mul_pi(m[7]);
  const qc u = A::sub(m[1], j5), u2 = A::add(m[1], j5);
  const qc v = A::sub(m[3], j7), v2 = A::add(m[3], j7);
  const qc l1 = A::mul_w(u, C16, -S16), l3 = A::mul_w(v, S16, -C16);
  const qc l3b = A::mul_w(u2, S16, -C16), l9 = A::mul_w(v2, -C16, S16);
  const qc qr = A::add(q, r), qmr = A::sub(q, r);
  const qc ls = A::add(l1, l3), ld = A::mul_mi(A::sub(l3, l1));
  y[1] = A::add(qr, ls);
  y[9] = A::sub(qr, ls);
  y[5] = A::sub(qmr, ld);
  y[13] = A::add(qmr, ld);
  const qc qa = A::sub(q2, r2), qb = A::add(q2, r2);
  const qc ls2 = A::add(l3b, l9), ld2 = A::mul_mi(A::sub(l9, l3b));
  y[3] = A::add(qa, ls2);
  y[11] = A::sub(qa, ls2);
  y[7] = A::sub(qb, ld2);
  y[15] = A::add(qb, ld2);
}

template <int R, int B>
__device__ __forceinline__ void q_dft(const qc* a, qc* y) {
  if constexpr (R == 1)
    y[0] = a[0];
  else if constexpr (R == 2)
    q_dft2<B>(a, y);
  else if constexpr (R == 4)
    q_dft4<B>(a, y);
  else if constexpr (R == 8)
    q_dft8<B>(a, y);
  else
    q_dft16<B>(a, y);
}

constexpr int ilog2_c(int r) { return r <= 1 ? 0 : 1 + ilog2_c(r / 2); }

// storage word <-> components (little endian: re in the low part)
__device__ __forceinline__ qc unpack(int w) { return {(w << 16) >> 16, w >> 16}; }
__device__ __forceinline__ qc unpack(short w) {
  const int v = w;
  return {(v << 24) >> 24, v >> 8};
}
// saturate both components to B bits and pack
template <int B>
__device__ __forceinline__ typename Fx<B>::W pack(qc v) {
  if constexpr (B == 16) {
    int d;
    asm("cvt.pack.sat.s16.s32 %0, %1, %2;" : "=r"(d) : "r"(v.im), "r"(v.re));
    return d;
  } else {
    const int re = max(-128, min(127, v.re)), im = max(-128, min(127, v.im));
    return short((re & 0xff) | (im << 8));
  }
}

template <int B>
__device__ __forceinline__ qc pre(qc v, int s) {
  return {rshr(v.re, s), rshr(v.im, s)};
}

// n <= 16: one thread per member
template <int N, int DIR, int B>
__global__ void __launch_bounds__(256) fx_small_kernel(const FixedLaunch L) {
  using W = typename Fx<B>::W;
  griddep_wait();  // launched programmatically (launch_pdl.cuh)
  griddep_launch_dependents();
  const int64_t b = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (b >= L.howmany) return;
  constexpr int S = ilog2_c(N);
  const W* x = static_cast<const W*>(L.in) + b * L.idist;
  W* y = static_cast<W*>(L.out) + b * L.odist;
  qc a[N], r[N];
#pragma unroll
  for (int k = 0; k < N; ++k) {
    const qc v = unpack(x[k * L.istride]);
    a[k] = S ? pre<B>(v, S) : v;
  }
  q_dft<N, B>(a, r);
#pragma unroll
  for (int k = 0; k < N; ++k) y[k * L.ostride] = pack<B>(r[DIR < 0 ? k : (N - k) % N]);
}

// padded shared-memory position of element k (16 columns per row, one
// spare word per row) and the member pitch (== 16 mod 32 words)
__host__ __device__ constexpr int fx_pos(int k) { return k + (k >> 4); }
__host__ __device__ constexpr int fx_pitch(int n) { return ((17 * (n / 16) + 15) / 32) * 32 + 16; }

// n = 16 m, m = 2..16: G = blockDim / 16 members per CTA
template <int N, int DIR, int B>
__global__ void __launch_bounds__(256) fx_two_stage_kernel(const FixedLaunch L) {
  using W = typename Fx<B>::W;
  griddep_wait();  // launched programmatically (launch_pdl.cuh)
  griddep_launch_dependents();
  constexpr int M = N / 16, SM = ilog2_c(M);
  constexpr int PITCH = fx_pitch(N);
  extern __shared__ __align__(16) unsigned char fsm[];
  short4* tw = reinterpret_cast<short4*>(fsm);  // (c, s, cvt(-s), c)
  W* tile = reinterpret_cast<W*>(tw + 15 * (M - 1 > 0 ? M - 1 : 1));
  const int G = blockDim.x / 16;
  const int64_t b0 = int64_t(blockIdx.x) * G;
  const int64_t left = L.howmany - b0;
  const int cnt = left < G ? int(left) : G;
  for (int i = threadIdx.x; i < 15 * (M - 1); i += blockDim.x) tw[i] = L.tw[i];
  const W* in = static_cast<const W*>(L.in);
  // stage the members (each thread: consecutive elements across members),
  // asynchronous copies so that all of a thread's loads are in flight
  for (int f = threadIdx.x; f < cnt * N; f += blockDim.x) {
    const int g = f / N, k = f - g * N;
    const W* src = in + (b0 + g) * L.idist + int64_t(k) * L.istride;
    if constexpr (B == 16)
      cp_async4(tile + g * PITCH + fx_pos(k), src);
    else
      tile[g * PITCH + fx_pos(k)] = *src;
  }
  cp_async_wait_all();
  __syncthreads();
  const int g = threadIdx.x >> 4, c = threadIdx.x & 15;
  W* mine = tile + g * PITCH;
  if (g < cnt) {  // stage 1: length-M codelet down column c, in place
    qc a[M], r[M];
#pragma unroll
    for (int q = 0; q < M; ++q) a[q] = pre<B>(unpack(mine[fx_pos(c + 16 * q)]), SM);
    q_dft<M, B>(a, r);
#pragma unroll
    for (int k = 0; k < M; ++k) mine[fx_pos(c + 16 * k)] = pack<B>(r[DIR < 0 ? k : (M - k) % M]);
  }
  __syncthreads();
  // stage 2: rows (member, j) spread over the CTA's threads
  for (int row = threadIdx.x; row < cnt * M; row += blockDim.x) {
    const int gg = row / M, j = row - gg * M;
    const W* src = tile + gg * PITCH + fx_pos(16 * j);
    qc a[16], r[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const qc s = pre<B>(unpack(src[i]), 4);
      a[i] = (i == 0 || j == 0) ? s : Ar<B>::twiddle(s, tw[15 * (j - 1) + (i - 1)]);
    }
    q_dft<16, B>(a, r);
    W* y = static_cast<W*>(L.out) + (b0 + gg) * L.odist;
#pragma unroll
    for (int k = 0; k < 16; ++k) y[int64_t(j + M * k) * L.ostride] = pack<B>(r[DIR < 0 ? k : (16 - k) & 15]);
  }
}

// n = 256 m', m' = 2..16: one member per CTA of 256 threads
template <int N, int DIR, int B>
__global__ void __launch_bounds__(256) fx_three_stage_kernel(const FixedLaunch L) {
  using W = typename Fx<B>::W;
  griddep_wait();  // launched programmatically (launch_pdl.cuh)
  griddep_launch_dependents();
  constexpr int M2 = N / 256, S2 = ilog2_c(M2), M = N / 16;
  extern __shared__ __align__(16) unsigned char fsm[];
  W* t = reinterpret_cast<W*>(fsm);
  const int64_t b = blockIdx.x;
  const W* x = static_cast<const W*>(L.in) + b * L.idist;
  W* y = static_cast<W*>(L.out) + b * L.odist;
  for (int k = threadIdx.x; k < N; k += 256) t[fx_pos(k)] = x[int64_t(k) * L.istride];
  __syncthreads();
  {  // length-M2 codelet down column c = threadIdx.x, in place
    const int c = threadIdx.x;
    qc a[M2], r[M2];
#pragma unroll
    for (int q = 0; q < M2; ++q) a[q] = pre<B>(unpack(t[fx_pos(c + 256 * q)]), S2);
    q_dft<M2, B>(a, r);
#pragma unroll
    for (int k = 0; k < M2; ++k) t[fx_pos(c + 256 * k)] = pack<B>(r[DIR < 0 ? k : (M2 - k) % M2]);
  }
  __syncthreads();
  // inner radix-16 level: task (row i0, column tc)
  const int i0 = threadIdx.x >> 4, tc = threadIdx.x & 15;
  const bool act = threadIdx.x < 16 * M2;
  qc r[16];
  if (act) {
    qc a[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const qc s = pre<B>(unpack(t[fx_pos(256 * i0 + tc + 16 * i)]), 4);
      a[i] = (i == 0 || i0 == 0) ? s : Ar<B>::twiddle(s, __ldg(L.tw2 + 15 * (i0 - 1) + (i - 1)));
    }
    q_dft<16, B>(a, r);
  }
  __syncthreads();  // every input of this level is read before any output lands
  if (act) {
#pragma unroll
    for (int k = 0; k < 16; ++k) t[fx_pos(16 * i0 + tc + 16 * M2 * k)] = pack<B>(r[DIR < 0 ? k : (16 - k) & 15]);
  }
  __syncthreads();
  // outer radix-16 level: row j
  if (threadIdx.x < M) {
    const int j = threadIdx.x;
    qc a[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const qc s = pre<B>(unpack(t[fx_pos(16 * j + i)]), 4);
      a[i] = (i == 0 || j == 0) ? s : Ar<B>::twiddle(s, __ldg(L.tw + 15 * (j - 1) + (i - 1)));
    }
    q_dft<16, B>(a, r);
#pragma unroll
    for (int k = 0; k < 16; ++k) y[int64_t(j + M * k) * L.ostride] = pack<B>(r[DIR < 0 ? k : (16 - k) & 15]);
  }
}

// ---- R2C (forward): the reference's real-input plans ----
// The reference's R2C plans run the C2C levels on the real input (imaginary
// parts zero) but each twiddled radix-16 level computes only the rows
// r <= rows/2 of its sub-spectra and writes row rows - r (r >= 1) as the
// conjugate of row r with the codelet outputs reversed (output k of row
// rows - r = conj(output 15 - k of row r): X[L - b] = conj(X[b]) for the
// length-L sub-spectrum of a real sequence; planner/strategies/
// cooley_tukey.hpp:145-248, 386-470).  The real-input codelets come in
// kernel variants that round differently at lengths 4 and 8
// (providers/aot/aot_kernel_data.cpp:188-252): the unit-output-distance ones
// (uu, gu: a batch of more than one member with odist 1, and the first stage
// of every larger plan) and the others (uun, us, gs).  Lengths 2 and 16,
// and length 4 of the unit-output-distance variants, are the complex codelet
// on (x, 0).  Outputs are bins 0..n/2.

// scalar storage of one real lane
template <int B>
using FxS = typename std::conditional<B == 16, short, signed char>::type;

template <int B>
__device__ __forceinline__ int fx_sat(int v) {
  return max(Fx<B>::LO, min(Fx<B>::HI, v));
}

// the reference's 8-point real-input codelet (forward), on raw reals.
// UO false (uun, us, gs): X2 = (rdm(p, 1), rdm(e1, -1)),
//   X1 = (rdm(d04 + rg, 1), rdm(d26 + rh, -1)), X3 = (d04 - rg, d26 - rh);
// UO true (uu, gu): X2 = (p, -rdm(e1, 1)),
//   X1 = (d04 + rg, -rdm(d26 + rh, 1)), X3 = (d04 - rg, rdm(d26 - rh, 1));
// rg, rh = rdm(g, c8), rdm(h, c8); 1 and -1 are the format's HI and LO.
// Every intermediate is within range after the 3-bit pre-shift, so the
// negations are exact.
template <int B, bool UO>
__device__ __forceinline__ void q_real8(const int* x, qc* y) {
  using A = Ar<B>;
  constexpr int C8 = Fx<B>::C8, HI = Fx<B>::HI, LO = Fx<B>::LO;
  int a[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = rshr(x[k], 3);
  const int d15 = fx_sat<B>(a[1] - a[5]), s15 = fx_sat<B>(a[1] + a[5]);
  const int d26 = fx_sat<B>(a[2] - a[6]), s26 = fx_sat<B>(a[2] + a[6]);
  const int d37 = fx_sat<B>(a[3] - a[7]), s37 = fx_sat<B>(a[3] + a[7]);
  const int d04 = fx_sat<B>(a[0] - a[4]), s04 = fx_sat<B>(a[0] + a[4]);
  const int e1 = fx_sat<B>(s15 - s37), f1 = fx_sat<B>(s15 + s37);
  const int g = fx_sat<B>(d15 - d37), h = fx_sat<B>(d15 + d37);
  const int rg = A::template rdm<C8>(g), rh = A::template rdm<C8>(h);
  const int p = fx_sat<B>(s04 - s26), q = fx_sat<B>(s04 + s26);
  y[0] = {fx_sat<B>(q + f1), 0};
  y[4] = {fx_sat<B>(q - f1), 0};
  if constexpr (UO) {
    y[2] = {p, -A::template rdm<HI>(e1)};
    y[1] = {fx_sat<B>(d04 + rg), -A::template rdm<HI>(fx_sat<B>(d26 + rh))};
    y[3] = {fx_sat<B>(d04 - rg), A::template rdm<HI>(fx_sat<B>(d26 - rh))};
  } else {
    y[2] = {A::template rdm<HI>(p), A::template rdm<LO>(e1)};
    y[1] = {A::template rdm<HI>(fx_sat<B>(d04 + rg)), A::template rdm<LO>(fx_sat<B>(d26 + rh))};
    y[3] = {fx_sat<B>(d04 - rg), fx_sat<B>(d26 - rh)};
  }
  y[5] = y[6] = y[7] = {0, 0};
}

// the 4-point real-input codelet of the uun / us / gs variants: X0, X2 as
// the complex codelet, X1 = (rdm(a0 - a2, 1), rdm(a1 - a3, -1))
template <int B>
__device__ __forceinline__ void q_real4(const int* x, qc* y) {
  using A = Ar<B>;
  int a[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) a[k] = rshr(x[k], 2);
  const int s02 = a[0] + a[2], d02 = a[0] - a[2], s13 = a[1] + a[3], d13 = a[1] - a[3];
  y[0] = {s02 + s13, 0};
  y[2] = {s02 - s13, 0};
  y[1] = {A::template rdm<Fx<B>::HI>(d02), A::template rdm<Fx<B>::LO>(d13)};
  y[3] = {0, 0};
}

// real-input codelet of length R on raw reals; UO selects the
// unit-output-distance variant
template <int R, int B, bool UO>
__device__ __forceinline__ void q_real_codelet(const int* x, qc* y) {
  if constexpr (R == 8) {
    q_real8<B, UO>(x, y);
  } else if constexpr (R == 4 && !UO) {
    q_real4<B>(x, y);
  } else {
    constexpr int S = ilog2_c(R);
    qc a[R];
#pragma unroll
    for (int k = 0; k < R; ++k) a[k] = {S ? rshr(x[k], S) : x[k], 0};
    q_dft<R, B>(a, y);
  }
}

template <int B>
__device__ __forceinline__ qc fx_conj(qc v) { return {v.re, -v.im}; }

// n <= 16: one thread per member
template <int N, int B, bool UO>
__global__ void __launch_bounds__(256) fx_r2c_small_kernel(const FixedLaunch L) {
  using W = typename Fx<B>::W;
  griddep_wait();  // launched programmatically (launch_pdl.cuh)
  griddep_launch_dependents();
  const int64_t b = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (b >= L.howmany) return;
  const FxS<B>* x = static_cast<const FxS<B>*>(L.in) + b * L.idist;
  W* y = static_cast<W*>(L.out) + b * L.odist;
  int xr[N];
  qc r[N];
#pragma unroll
  for (int k = 0; k < N; ++k) xr[k] = x[k * L.istride];
  q_real_codelet<N, B, UO>(xr, r);
#pragma unroll
  for (int k = 0; k <= N / 2; ++k) y[k * L.ostride] = pack<B>(r[k]);
}

// R2C two-stage kernel geometry: 256 threads, G members per CTA so that the
// row stage gives every thread one row (rows j <= M/2 of each member).
// Shared memory: twiddles, the column-stage outputs (rows 0..M/2 only, one
// pad word per 16-word row), then (16-byte aligned) the real inputs, RP
// lanes per member; after the column stage that area holds the members'
// output bins, H = N/2 + 1 words apart (G H words of W fit in G RP lanes
// of S since 2 (N/2 + 1) <= N + 16).
__host__ __device__ constexpr int fx_r2c_rows(int n) { return n / 32 + 1; }
__host__ __device__ constexpr int fx_r2c_members(int n) { return 256 / fx_r2c_rows(n); }
__host__ __device__ constexpr int fx_r2c_pitch(int n) { return ((17 * fx_r2c_rows(n) + 15) / 32) * 32 + 16; }
__host__ __device__ constexpr int fx_r2c_rpitch(int n) { return n + 16; }
template <int B>
__host__ __device__ constexpr int fx_r2c_real_offset(int n) {
  return (8 * 15 * (n / 16 - 1 > 0 ? n / 16 - 1 : 1) +
          int(sizeof(typename Fx<B>::W)) * fx_r2c_members(n) * fx_r2c_pitch(n) + 15) /
         16 * 16;
}
template <int B>
__host__ __device__ constexpr int fx_r2c_smem_bytes(int n) {
  return fx_r2c_real_offset<B>(n) + fx_r2c_members(n) * fx_r2c_rpitch(n) * int(sizeof(FxS<B>));
}

// n = 16 m, m = 2..16.  Inputs arrive by 16-byte loads when the members are
// 16-byte aligned rows (unit istride); outputs leave as coalesced runs of
// each member's bins.
template <int N, int B>
__global__ void __launch_bounds__(256) fx_r2c_two_stage_kernel(const FixedLaunch L) {
  using W = typename Fx<B>::W;
  using S = FxS<B>;
  griddep_wait();  // launched programmatically (launch_pdl.cuh)
  griddep_launch_dependents();
  constexpr int M = N / 16, ROWS = fx_r2c_rows(N), G = fx_r2c_members(N), PITCH = fx_r2c_pitch(N);
  constexpr int H = N / 2 + 1, RP = fx_r2c_rpitch(N);
  static_assert(ROWS == M / 2 + 1 && G * ROWS <= 256, "geometry");
  extern __shared__ __align__(16) unsigned char fsm[];
  short4* tw = reinterpret_cast<short4*>(fsm);  // (c, s, cvt(-s), c)
  W* tile = reinterpret_cast<W*>(tw + 15 * (M - 1 > 0 ? M - 1 : 1));
  S* rin = reinterpret_cast<S*>(fsm + fx_r2c_real_offset<B>(N));
  W* bins = reinterpret_cast<W*>(rin);
  const int64_t b0 = int64_t(blockIdx.x) * G;
  const int64_t left = L.howmany - b0;
  const int cnt = left < G ? int(left) : G;
  for (int i = threadIdx.x; i < 15 * (M - 1); i += 256) tw[i] = L.tw[i];
  const S* in = static_cast<const S*>(L.in);
  constexpr int VPM = N * int(sizeof(S)) / 16;  // 16-byte vectors per member row
  const bool vec = L.istride == 1 && (L.idist * int64_t(sizeof(S))) % 16 == 0 &&
                   (reinterpret_cast<uintptr_t>(in) & 15) == 0;
  if (vec) {
    for (int f = threadIdx.x; f < cnt * VPM; f += 256) {
      const int g = f / VPM, v = f - g * VPM;
      const uint4 d = __ldg(reinterpret_cast<const uint4*>(in + (b0 + g) * L.idist) + v);
      *reinterpret_cast<uint4*>(rin + g * RP + v * (16 / int(sizeof(S)))) = d;
    }
  } else {
    for (int f = threadIdx.x; f < cnt * N; f += 256) {
      const int g = f / N, k = f - g * N;
      rin[g * RP + k] = in[(b0 + g) * L.idist + int64_t(k) * L.istride];
    }
  }
  __syncthreads();
  // stage 1: length-M real codelet down column c of member g; only the
  // bins k <= M/2 are kept (the rows stage 2 reads)
  for (int task = threadIdx.x; task < cnt * 16; task += 256) {
    const int g = task >> 4, c = task & 15;
    int xr[M];
    qc r[M];
#pragma unroll
    for (int q = 0; q < M; ++q) xr[q] = rin[g * RP + c + 16 * q];
    q_real_codelet<M, B, true>(xr, r);
    W* mine = tile + g * PITCH;
#pragma unroll
    for (int k = 0; k < ROWS; ++k) mine[fx_pos(c + 16 * k)] = pack<B>(r[k]);
  }
  __syncthreads();
  // stage 2: rows (member, j <= M/2); row M - j is the mirror of row j.
  // Bins go to the shared output area (the real inputs are consumed).
  for (int row = threadIdx.x; row < cnt * ROWS; row += 256) {
    const int gg = row / ROWS, j = row - gg * ROWS;
    const W* src = tile + gg * PITCH + fx_pos(16 * j);
    qc a[16], r[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const qc s = pre<B>(unpack(src[i]), 4);
      a[i] = (i == 0 || j == 0) ? s : Ar<B>::twiddle(s, tw[15 * (j - 1) + (i - 1)]);
    }
    q_dft<16, B>(a, r);
    W* y = bins + gg * H;
    const bool mirror = j > 0 && 2 * j < M;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const int t = j + M * k, tm = (M - j) + M * (15 - k);
      if (t <= N / 2) y[t] = pack<B>(r[k]);
      if (mirror && tm <= N / 2) y[tm] = pack<B>(fx_conj<B>(r[k]));
    }
  }
  __syncthreads();
  W* out = static_cast<W*>(L.out);
  for (int f = threadIdx.x; f < cnt * H; f += 256) {
    const int gg = f / H, t = f - gg * H;
    out[(b0 + gg) * L.odist + int64_t(t) * L.ostride] = bins[gg * H + t];
  }
}

// n = 256 m', m' = 2..16: one member per CTA of 256 threads
template <int N, int B>
__global__ void __launch_bounds__(256) fx_r2c_three_stage_kernel(const FixedLaunch L) {
  using W = typename Fx<B>::W;
  griddep_wait();  // launched programmatically (launch_pdl.cuh)
  griddep_launch_dependents();
  constexpr int M2 = N / 256, M = N / 16;
  extern __shared__ __align__(16) unsigned char fsm[];
  W* t = reinterpret_cast<W*>(fsm);
  const int64_t b = blockIdx.x;
  const FxS<B>* x = static_cast<const FxS<B>*>(L.in) + b * L.idist;
  W* y = static_cast<W*>(L.out) + b * L.odist;
  for (int k = threadIdx.x; k < N; k += 256) t[fx_pos(k)] = pack<B>(qc{x[int64_t(k) * L.istride], 0});
  __syncthreads();
  {  // length-M2 real codelet down column c = threadIdx.x, in place
    const int c = threadIdx.x;
    int xr[M2];
    qc r[M2];
#pragma unroll
    for (int q = 0; q < M2; ++q) xr[q] = unpack(t[fx_pos(c + 256 * q)]).re;
    q_real_codelet<M2, B, true>(xr, r);
#pragma unroll
    for (int k = 0; k < M2; ++k) t[fx_pos(c + 256 * k)] = pack<B>(r[k]);
  }
  __syncthreads();
  // inner radix-16 level: task (row i0 <= M2/2, column tc); row M2 - i0 is
  // the mirror of row i0
  const int i0 = threadIdx.x >> 4, tc = threadIdx.x & 15;
  const bool act = i0 <= M2 / 2;
  qc r[16];
  if (act) {
    qc a[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const qc s = pre<B>(unpack(t[fx_pos(256 * i0 + tc + 16 * i)]), 4);
      a[i] = (i == 0 || i0 == 0) ? s : Ar<B>::twiddle(s, __ldg(L.tw2 + 15 * (i0 - 1) + (i - 1)));
    }
    q_dft<16, B>(a, r);
  }
  __syncthreads();  // every input of this level is read before any output lands
  if (act) {
    const bool mirror = i0 > 0 && 2 * i0 < M2;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      t[fx_pos(16 * i0 + tc + 16 * M2 * k)] = pack<B>(r[k]);
      if (mirror) t[fx_pos(16 * (M2 - i0) + tc + 16 * M2 * (15 - k))] = pack<B>(fx_conj<B>(r[k]));
    }
  }
  __syncthreads();
  // outer radix-16 level: rows j <= M/2, row M - j the mirror of row j
  if (threadIdx.x <= M / 2) {
    const int j = threadIdx.x;
    qc a[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const qc s = pre<B>(unpack(t[fx_pos(16 * j + i)]), 4);
      a[i] = (i == 0 || j == 0) ? s : Ar<B>::twiddle(s, __ldg(L.tw + 15 * (j - 1) + (i - 1)));
    }
    q_dft<16, B>(a, r);
    const bool mirror = j > 0 && 2 * j < M;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const int tt = j + M * k, tm = (M - j) + M * (15 - k);
      if (tt <= N / 2) y[int64_t(tt) * L.ostride] = pack<B>(r[k]);
      if (mirror && tm <= N / 2) y[int64_t(tm) * L.ostride] = pack<B>(fx_conj<B>(r[k]));
    }
  }
}

bool fixed_supported(int64_t n) { return n >= 1 && n <= 4096 && (n & (n - 1)) == 0; }

template <int B>
static int fx_smem_bytes(int n, int members) {
  using W = typename Fx<B>::W;
  if (n <= 16) return 0;
  if (n > 256) return int(sizeof(W)) * (n + n / 16);
  return 8 * 15 * (n / 16 - 1 > 0 ? n / 16 - 1 : 1) + int(sizeof(W)) * members * fx_pitch(n);
}

template <int N, int DIR, int B>
static cudaError_t run_fx(const FixedLaunch& L, cudaStream_t st) {
  if constexpr (N <= 16) {
    const int64_t blocks = (L.howmany + 255) / 256;
    return launch_pdl(fx_small_kernel<N, DIR, B>, dim3(unsigned(blocks)), dim3(256), 0, st, L);
  } else if constexpr (N <= 256) {
    constexpr int kThreads = 256, G = kThreads / 16;
    const int smem = fx_smem_bytes<B>(N, G);
    const int64_t blocks = (L.howmany + G - 1) / G;
    return launch_pdl(fx_two_stage_kernel<N, DIR, B>, dim3(unsigned(blocks)), dim3(kThreads), size_t(smem), st, L);
  } else {
    const int smem = fx_smem_bytes<B>(N, 1);
    return launch_pdl(fx_three_stage_kernel<N, DIR, B>, dim3(unsigned(L.howmany)), dim3(256), size_t(smem), st, L);
  }
}

template <int N, int B>
static cudaError_t run_fx_r2c(const FixedLaunch& L, cudaStream_t st) {
  if constexpr (N <= 16) {
    const int64_t blocks = (L.howmany + 255) / 256;
    if (L.howmany > 1 && L.odist == 1)
      return launch_pdl(fx_r2c_small_kernel<N, B, true>, dim3(unsigned(blocks)), dim3(256), 0, st, L);
    return launch_pdl(fx_r2c_small_kernel<N, B, false>, dim3(unsigned(blocks)), dim3(256), 0, st, L);
  } else if constexpr (N <= 256) {
    constexpr int G = fx_r2c_members(N), smem = fx_r2c_smem_bytes<B>(N);
    static_assert(smem <= 48 * 1024, "default dynamic shared-memory limit");
    const int64_t blocks = (L.howmany + G - 1) / G;
    return launch_pdl(fx_r2c_two_stage_kernel<N, B>, dim3(unsigned(blocks)), dim3(256), size_t(smem), st, L);
  } else {
    const int smem = fx_smem_bytes<B>(N, 1);
    return launch_pdl(fx_r2c_three_stage_kernel<N, B>, dim3(unsigned(L.howmany)), dim3(256), size_t(smem), st, L);
  }
}

template <int B>
static cudaError_t launch_fx_r2c(int n, const FixedLaunch& L, cudaStream_t st) {
  switch (n) {
    case 2: return run_fx_r2c<2, B>(L, st);
    case 4: return run_fx_r2c<4, B>(L, st);
    case 8: return run_fx_r2c<8, B>(L, st);
    case 16: return run_fx_r2c<16, B>(L, st);
    case 32: return run_fx_r2c<32, B>(L, st);
    case 64: return run_fx_r2c<64, B>(L, st);
    case 128: return run_fx_r2c<128, B>(L, st);
    case 256: return run_fx_r2c<256, B>(L, st);
    case 512: return run_fx_r2c<512, B>(L, st);
    case 1024: return run_fx_r2c<1024, B>(L, st);
    case 2048: return run_fx_r2c<2048, B>(L, st);
    case 4096: return run_fx_r2c<4096, B>(L, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_fixed_r2c(int bits, int n, const FixedLaunch& L, cudaStream_t st) {
  if (L.howmany > 0x7fffffffLL && n > 256) return cudaErrorInvalidValue;  // one CTA per member
  return bits == 16 ? launch_fx_r2c<16>(n, L, st) : launch_fx_r2c<8>(n, L, st);
}

// ---- C2R (backward): the reference's real-output plans ----
// The C2R plan runs the decomposition backward with decimation in frequency
// (planner/strategies/cooley_tukey.hpp:250-323, 498-580): a radix-16 DIF
// level over rows j = 0..m/2 of the Hermitian input (row j takes
// X[j + m i], the ones past the stored half as conjugates of
// X[m (16 - i) - j]; a backward 16-point codelet; outputs k >= 1 of rows
// j >= 1 times W_N^{jk}), then per column a real-output codelet of length
// m (n <= 256) or a second such level over m/16 rows and real-output
// codelets of length m/16 on 256 lanes (n >= 512).  Inputs are pre-shifted
// by log2 of the codelet length, then conjugated as products by
// (1 - 2^-(B-1), -1).  The real-output codelets of lengths 2 and 4 are the
// backward codelet's real parts; those of 8 and 16 round their constant
// products in their own places (cr_real8, cr_real16).  The operands here
// reach the full lane range, so every add saturates and every MAC wraps at
// 2B bits, as the reference's sqadd / smlal lanes do.

template <int B>
__device__ __forceinline__ int cr_add(int a, int b) { return fx_sat<B>(a + b); }
template <int B>
__device__ __forceinline__ int cr_sub(int a, int b) { return fx_sat<B>(a - b); }
// a times the constant k, one rounding, saturated
template <int B>
__device__ __forceinline__ int cr_rdm(int a, int k) { return fx_sat<B>((a * k + (1 << (B - 2))) >> (B - 1)); }
// two products accumulated in a 2B-bit lane (wrapping), one rounding narrow
template <int B>
__device__ __forceinline__ int cr_mac2(int a, int ka, int b, int kb) {
  const unsigned u = unsigned(a) * unsigned(ka) + unsigned(b) * unsigned(kb);
  const int64_t acc = B == 16 ? int64_t(int(u)) : int64_t(short(u & 0xffffu));
  return fx_sat<B>(int((acc + (1 << (B - 2))) >> (B - 1)));
}
// pre-shifted input, conjugated by the constant products when asked
template <int B>
__device__ __forceinline__ qc cr_in(qc v, int s, bool conj) {
  const qc a = s ? qc{rshr(v.re, s), rshr(v.im, s)} : v;
  return conj ? qc{cr_rdm<B>(a.re, Fx<B>::HI), cr_rdm<B>(a.im, Fx<B>::LO)} : a;
}

// real-output codelet of length 8 on the extended, pre-shifted inputs A
template <int B>
__device__ __forceinline__ void cr_real8(const qc* A, int* x) {
  constexpr int C8 = Fx<B>::C8;
  const int s04 = cr_add<B>(A[0].re, A[4].re), d04 = cr_sub<B>(A[0].re, A[4].re);
  const int s26 = cr_add<B>(A[2].re, A[6].re), e26 = cr_sub<B>(A[2].im, A[6].im);
  const qc p15 = {cr_sub<B>(A[1].re, A[5].re), cr_sub<B>(A[1].im, A[5].im)};
  const qc p37 = {cr_sub<B>(A[3].re, A[7].re), cr_sub<B>(A[3].im, A[7].im)};
  const int qr = cr_add<B>(cr_add<B>(A[1].re, A[5].re), cr_add<B>(A[3].re, A[7].re));
  const int qi = cr_sub<B>(cr_add<B>(A[1].im, A[5].im), cr_add<B>(A[3].im, A[7].im));
  const int u = cr_rdm<B>(cr_sub<B>(p15.re, p37.re), C8);
  const int v = cr_rdm<B>(cr_add<B>(p15.im, p37.im), C8);
  const int e = cr_add<B>(s04, s26), g = cr_sub<B>(s04, s26);
  const int a = cr_add<B>(d04, u), b = cr_sub<B>(fx_sat<B>(-e26), v);
  const int c = cr_sub<B>(d04, u), d = cr_sub<B>(v, e26);
  x[0] = cr_add<B>(e, qr);
  x[4] = cr_sub<B>(e, qr);
  x[2] = cr_sub<B>(g, qi);
  x[6] = cr_add<B>(g, qi);
  x[1] = cr_add<B>(a, b);
  x[7] = cr_sub<B>(a, b);
  x[3] = cr_sub<B>(c, d);
  x[5] = cr_add<B>(c, d);
}

// real-output codelet of length 16 on the extended, pre-shifted inputs A
template <int B>
__device__ __forceinline__ void cr_real16(const qc* A, int* x) {
  constexpr int C8 = Fx<B>::C8, C16 = Fx<B>::C16, S16 = Fx<B>::S16, HI = Fx<B>::HI, LO = Fx<B>::LO;
  auto ad = [](int a, int b) { return cr_add<B>(a, b); };
  auto sb = [](int a, int b) { return cr_sub<B>(a, b); };
  auto rd = [](int a, int k) { return cr_rdm<B>(a, k); };
  auto mc = [](int a, int ka, int b, int kb) { return cr_mac2<B>(a, ka, b, kb); };
  // even half: inputs 0, 2, ..., 14
  const int s08 = ad(A[0].re, A[8].re), d08 = sb(A[0].re, A[8].re);
  const int s4c = ad(A[4].re, A[12].re), d4c = sb(A[4].im, A[12].im);
  const int ev = ad(s08, s4c), ew = sb(s08, s4c);
  const int s2a6e = ad(ad(A[2].re, A[10].re), ad(A[6].re, A[14].re));
  const int r2a = sb(A[2].re, A[10].re), i2a = sb(A[2].im, A[10].im);
  const int r6e = sb(A[6].re, A[14].re), i6e = sb(A[6].im, A[14].im);
  const int i26 = sb(ad(A[2].im, A[10].im), ad(A[6].im, A[14].im));
  const int e0 = ad(ev, s2a6e), e4 = sb(ev, s2a6e);
  const int f1 = sb(d08, d4c), f3 = ad(d08, d4c);
  const int f2 = sb(ew, i26), f6 = ad(ew, i26);
  // odd half: inputs 1, 3, ..., 15
  const int s19 = ad(A[1].re, A[9].re), s5d = ad(A[5].re, A[13].re);
  const int s3b = ad(A[3].re, A[11].re), s7f = ad(A[7].re, A[15].re);
  const int o0 = ad(ad(s19, s5d), ad(s3b, s7f));
  const int i3b = sb(A[3].im, A[11].im), r7f = rd(sb(A[7].re, A[15].re), HI);
  const int r3b = sb(A[3].re, A[11].re), i7f = rd(sb(A[7].im, A[15].im), LO);
  const int i19 = sb(A[1].im, A[9].im), r5d = rd(sb(A[5].re, A[13].re), HI);
  const int r19 = sb(A[1].re, A[9].re), i5d = rd(sb(A[5].im, A[13].im), LO);
  const int p3 = ad(i3b, r7f), q3 = ad(r3b, i7f), p1 = ad(i19, r5d), q1 = ad(r19, i5d);
  const int m3 = sb(i3b, r7f), n3 = sb(r3b, i7f), m1 = sb(i19, r5d), n1 = sb(r19, i5d);
  const int j3b = ad(A[3].im, A[11].im), j7f = ad(A[7].im, A[15].im), j37 = sb(j3b, j7f);
  const int k37 = sb(s3b, s7f);
  const int j19 = ad(A[1].im, A[9].im), j5d = ad(A[5].im, A[13].im), j15 = sb(j19, j5d);
  const int k15 = sb(s19, s5d);
  const int o4 = sb(ad(j19, j5d), ad(j3b, j7f));
  // rotations
  const int w1 = rd(sb(mc(i6e, -C8, rd(r6e, -C8), HI), mc(i2a, C8, rd(r2a, C8), LO)), LO);
  const int w3 = ad(mc(r2a, C8, rd(i2a, C8), HI), mc(r6e, -C8, rd(i6e, -C8), LO));
  const int z2 = rd(sb(mc(j37, -C8, rd(k37, -C8), HI), mc(j15, C8, rd(k15, C8), LO)), LO);
  const int z6 = ad(mc(k15, C8, rd(j15, C8), HI), mc(k37, -C8, rd(j37, -C8), LO));
  const int z1 = rd(sb(mc(p3, -C16, q3, S16), mc(p1, S16, q1, -C16)), LO);
  const int z3 = rd(sb(mc(m3, S16, n3, -C16), mc(m1, C16, n1, -S16)), LO);
  const int z5 = ad(mc(q1, S16, p1, C16), mc(q3, -C16, p3, -S16));
  const int z7 = ad(mc(n1, C16, m1, S16), mc(n3, S16, m3, C16));
  const int g1 = sb(f1, w1), g5 = ad(f1, w1), g3 = sb(f3, w3), g7 = ad(f3, w3);
  x[0] = ad(e0, o0);
  x[8] = sb(e0, o0);
  x[4] = sb(e4, o4);
  x[12] = ad(e4, o4);
  x[2] = sb(f2, z2);
  x[10] = ad(f2, z2);
  x[6] = sb(f6, z6);
  x[14] = ad(f6, z6);
  x[1] = sb(g1, z1);
  x[9] = ad(g1, z1);
  x[3] = sb(g3, z3);
  x[11] = ad(g3, z3);
  x[5] = sb(g5, z5);
  x[13] = ad(g5, z5);
  x[7] = sb(g7, z7);
  x[15] = ad(g7, z7);
}

// real-output codelet of length R over the stored half get(e), e = 0..R/2
template <int R, int B, class Get>
__device__ __forceinline__ void cr_real_out(Get get, int* x) {
  constexpr int S = ilog2_c(R);
  qc A[R];
#pragma unroll
  for (int i = 0; i < R; ++i) A[i] = i <= R / 2 ? cr_in<B>(get(i), S, false) : cr_in<B>(get(R - i), S, true);
  if constexpr (R == 8) {
    cr_real8<B>(A, x);
  } else if constexpr (R == 16) {
    cr_real16<B>(A, x);
  } else {
    qc y[R];
    q_dft<R, B>(A, y);
#pragma unroll
    for (int k = 0; k < R; ++k) x[k] = fx_sat<B>(y[(R - k) % R].re);  // backward: forward output R - k
  }
}

// row j of a radix-16 DIF level over ROWS_ rows of a Hermitian sequence of
// length 16 rows (stored half get(e), e = 0..8 rows): 16 outputs, those
// k >= 1 of rows j >= 1 times the row's twiddle tw[15 (j - 1) + k - 1]
template <int B, class Get>
__device__ __forceinline__ void cr_dif_row(Get get, int rows, int j, const short4* tw, qc* out) {
  qc a[16], t[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    const bool direct = j == 0 ? i <= 8 : i <= 7;
    a[i] = cr_in<B>(get(direct ? j + rows * i : rows * (16 - i) - j), 4, !direct);
  }
  q_dft<16, B>(a, t);
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const qc v = {fx_sat<B>(t[(16 - k) & 15].re), fx_sat<B>(t[(16 - k) & 15].im)};  // backward output k
    if (j > 0 && k > 0) {
      const short4 w = __ldg(tw + 15 * (j - 1) + (k - 1));  // (c, s, cvt(-s), c)
      out[k] = {cr_mac2<B>(v.re, w.x, v.im, w.z), cr_mac2<B>(v.re, w.y, v.im, w.w)};
    } else {
      out[k] = v;
    }
  }
}

// n <= 16: one thread per member
template <int N, int B>
__global__ void __launch_bounds__(256) fx_c2r_small_kernel(const FixedLaunch L) {
  using W = typename Fx<B>::W;
  griddep_wait();  // launched programmatically (launch_pdl.cuh)
  griddep_launch_dependents();
  const int64_t b = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (b >= L.howmany) return;
  const W* X = static_cast<const W*>(L.in) + b * L.idist;
  FxS<B>* y = static_cast<FxS<B>*>(L.out) + b * L.odist;
  qc h[N / 2 + 1];
#pragma unroll
  for (int k = 0; k <= N / 2; ++k) h[k] = unpack(X[k * L.istride]);
  int x[N];
  cr_real_out<N, B>([&](int e) { return h[e]; }, x);
#pragma unroll
  for (int t = 0; t < N; ++t) y[t * L.ostride] = FxS<B>(x[t]);
}

// shared-memory layout of the C2R kernels: the members' stored halves
// (H words each), the first level's rows 0..m/2 (16 words each), [the
// second level's rows 0..m'/2 (256 words each)], the output reals
template <int B>
__host__ __device__ constexpr int cr_align16(int bytes) { return (bytes + 15) / 16 * 16; }
template <int N, int B>
struct CrSmem {
  static constexpr int H = N / 2 + 1, M = N / 16, ROWS = M / 2 + 1;
  static constexpr int M2 = N > 256 ? N / 256 : 0, ROWS2 = M2 / 2 + 1;
  static constexpr int G = N > 256 ? 1 : 16;  // members per CTA
  static constexpr int WB = int(sizeof(typename Fx<B>::W));
  static constexpr int X_OFF = 0;
  static constexpr int B_OFF = cr_align16<B>(X_OFF + G * H * WB);
  static constexpr int C_OFF = cr_align16<B>(B_OFF + G * ROWS * 16 * WB);
  static constexpr int O_OFF = cr_align16<B>(C_OFF + (M2 ? ROWS2 * 256 * WB : 0));
  static constexpr int BYTES = cr_align16<B>(O_OFF + G * N * int(sizeof(FxS<B>)));
};

// n = 16 m (m = 2..16, 16 members per CTA) or n = 256 m' (m' = 2..16, one
// member per CTA); 256 threads
template <int N, int B>
__global__ void __launch_bounds__(256) fx_c2r_kernel(const FixedLaunch L) {
  using W = typename Fx<B>::W;
  using Sm = CrSmem<N, B>;
  constexpr int H = Sm::H, M = Sm::M, ROWS = Sm::ROWS, M2 = Sm::M2, ROWS2 = Sm::ROWS2, G = Sm::G;
  griddep_wait();  // launched programmatically (launch_pdl.cuh)
  griddep_launch_dependents();
  extern __shared__ __align__(16) unsigned char fsm[];
  W* xs = reinterpret_cast<W*>(fsm + Sm::X_OFF);
  W* bs = reinterpret_cast<W*>(fsm + Sm::B_OFF);
  W* cs = reinterpret_cast<W*>(fsm + Sm::C_OFF);
  FxS<B>* os = reinterpret_cast<FxS<B>*>(fsm + Sm::O_OFF);
  const int64_t b0 = int64_t(blockIdx.x) * G;
  const int64_t left = L.howmany - b0;
  const int cnt = left < G ? int(left) : G;
  const W* X = static_cast<const W*>(L.in);
  for (int f = threadIdx.x; f < cnt * H; f += blockDim.x) {
    const int g = f / H, e = f - g * H;
    xs[f] = X[(b0 + g) * L.idist + int64_t(e) * L.istride];
  }
  __syncthreads();
  // first level: rows j = 0..m/2 of each member
  for (int task = threadIdx.x; task < cnt * ROWS; task += blockDim.x) {
    const int g = task / ROWS, j = task - g * ROWS;
    const W* src = xs + g * H;
    qc r[16];
    cr_dif_row<B>([&](int e) { return unpack(src[e]); }, M, j, L.tw, r);
    W* dst = bs + (g * ROWS + j) * 16;
#pragma unroll
    for (int k = 0; k < 16; ++k) dst[k] = pack<B>(r[k]);
  }
  __syncthreads();
  if constexpr (M2 == 0) {
    // real-output codelets of length m down the 16 columns
    for (int task = threadIdx.x; task < cnt * 16; task += blockDim.x) {
      const int g = task >> 4, k = task & 15;
      const W* col = bs + g * ROWS * 16 + k;
      int x[M];
      cr_real_out<M, B>([&](int e) { return unpack(col[16 * e]); }, x);
#pragma unroll
      for (int t = 0; t < M; ++t) os[g * N + k + 16 * t] = FxS<B>(x[t]);
    }
  } else {
    // second level: rows i = 0..m'/2 of each column's length-m sequence
    for (int task = threadIdx.x; task < 16 * ROWS2; task += blockDim.x) {
      const int k = task / ROWS2, i = task - k * ROWS2;
      qc r[16];
      cr_dif_row<B>([&](int e) { return unpack(bs[16 * e + k]); }, M2, i, L.tw2, r);
#pragma unroll
      for (int q = 0; q < 16; ++q) cs[256 * i + 16 * q + k] = pack<B>(r[q]);
    }
    __syncthreads();
    // real-output codelets of length m' on the 256 lanes
    for (int l = threadIdx.x; l < 256; l += blockDim.x) {
      int x[M2];
      cr_real_out<M2, B>([&](int e) { return unpack(cs[256 * e + l]); }, x);
#pragma unroll
      for (int t = 0; t < M2; ++t) os[l + 256 * t] = FxS<B>(x[t]);
    }
  }
  __syncthreads();
  FxS<B>* y = static_cast<FxS<B>*>(L.out);
  for (int f = threadIdx.x; f < cnt * N; f += blockDim.x) {
    const int g = f / N, t = f - g * N;
    y[(b0 + g) * L.odist + int64_t(t) * L.ostride] = os[f];
  }
}

template <int N, int B>
static cudaError_t run_fx_c2r(const FixedLaunch& L, cudaStream_t st) {
  if constexpr (N <= 16) {
    const int64_t blocks = (L.howmany + 255) / 256;
    return launch_pdl(fx_c2r_small_kernel<N, B>, dim3(unsigned(blocks)), dim3(256), 0, st, L);
  } else {
    using Sm = CrSmem<N, B>;
    static_assert(Sm::BYTES <= 48 * 1024, "default dynamic shared-memory limit");
    const int64_t blocks = (L.howmany + Sm::G - 1) / Sm::G;
    return launch_pdl(fx_c2r_kernel<N, B>, dim3(unsigned(blocks)), dim3(256), size_t(Sm::BYTES), st, L);
  }
}

template <int B>
static cudaError_t launch_fx_c2r(int n, const FixedLaunch& L, cudaStream_t st) {
  switch (n) {
    case 2: return run_fx_c2r<2, B>(L, st);
    case 4: return run_fx_c2r<4, B>(L, st);
    case 8: return run_fx_c2r<8, B>(L, st);
    case 16: return run_fx_c2r<16, B>(L, st);
    case 32: return run_fx_c2r<32, B>(L, st);
    case 64: return run_fx_c2r<64, B>(L, st);
    case 128: return run_fx_c2r<128, B>(L, st);
    case 256: return run_fx_c2r<256, B>(L, st);
    case 512: return run_fx_c2r<512, B>(L, st);
    case 1024: return run_fx_c2r<1024, B>(L, st);
    case 2048: return run_fx_c2r<2048, B>(L, st);
    case 4096: return run_fx_c2r<4096, B>(L, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_fixed_c2r(int bits, int n, const FixedLaunch& L, cudaStream_t st) {
  if (L.howmany > 0x7fffffffLL && n > 256) return cudaErrorInvalidValue;  // one CTA per member
  return bits == 16 ? launch_fx_c2r<16>(n, L, st) : launch_fx_c2r<8>(n, L, st);
}

template <int B>
static cudaError_t launch_fx(int n, int dir, const FixedLaunch& L, cudaStream_t st) {
#define PLFFT_B200_FX(NV) \
  if (n == NV) return dir < 0 ? run_fx<NV, -1, B>(L, st) : run_fx<NV, 1, B>(L, st);
  PLFFT_B200_FX(1)
  PLFFT_B200_FX(2)
  PLFFT_B200_FX(4)
  PLFFT_B200_FX(8)
  PLFFT_B200_FX(16)
  PLFFT_B200_FX(32)
  PLFFT_B200_FX(64)
  PLFFT_B200_FX(128)
  PLFFT_B200_FX(256)
  PLFFT_B200_FX(512)
  PLFFT_B200_FX(1024)
  PLFFT_B200_FX(2048)
  PLFFT_B200_FX(4096)
#undef PLFFT_B200_FX
  return cudaErrorInvalidValue;
}

cudaError_t launch_fixed(int bits, int n, int dir, const FixedLaunch& L, cudaStream_t st) {
  if (L.howmany > 0x7fffffffLL && n > 256) return cudaErrorInvalidValue;  // one CTA per member
  return bits == 16 ? launch_fx<16>(n, dir, L, st) : launch_fx<8>(n, dir, L, st);
}

}  // namespace plfft_b200
