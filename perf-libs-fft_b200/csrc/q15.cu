// Q0.15 fixed-point C2C for power-of-two n <= 256, bit-exact to the
// reference's NEON fixed-point path.
//
// Arithmetic (reference src/providers/jit/print_algo.cpp:1228-1230,
// src/providers/jit/emit.hpp:150-175 and :370-425, constant lowering
// print_algo.cpp:2150-2290): codelet inputs are pre-scaled by a rounding
// shift right by log2(radix); additions saturate to int16; a real-constant
// multiply is the rounding doubling high half (2 a k + 2^15) >> 16; a
// twiddle product is two 16x16 products accumulated in 32 bits (wrapping)
// and narrowed by one rounding, saturating shift by 15.  The codelets are
// radix 2, 4, 8 and the fixed-point split-radix 16
// (src/providers/jit/split_radix_z16.cpp, src/providers/jit/wfta_nfact.cpp:
// 89-97); a backward codelet of length r yields the forward codelet's
// output r-k at index k.  Decomposition for n = 16 m (the reference's
// ESTIMATE plan, src/planner/strategies/cooley_tukey.hpp:622-748): length-m
// codelets down the 16 columns x[c + 16 q], then per row j a 16-point
// codelet whose inputs i >= 1 are multiplied by the stored twiddle pair of
// W_n^{dir i j} (src/generate_twiddles.hpp:72-132), output y[j + m k].
//
// GPU mapping: a CTA takes G members; each member's n values are staged in
// shared memory at padded position k + k/16 (so a column and a row are both
// read without bank conflicts, and two members in one warp use disjoint
// banks), 16 threads run the column codelets in place, then one thread per
// row runs the twiddled 16-point codelet and stores its 16 outputs.
#include <stdint.h>

#include "kernels.h"
#include "launch_pdl.cuh"
#include "ptx.cuh"

namespace plfft_b200 {

struct qc {
  int re, im;
};

__device__ __forceinline__ int rshr(int v, int s) { return (v + (1 << (s - 1))) >> s; }
// sqrdmulh by a constant k, |k| <= 32767: never overflows or saturates
template <int K>
__device__ __forceinline__ int rdm(int a) {
  static_assert(K > -32768 && K <= 32767, "constant out of range");
  return (2 * a * K + 32768) >> 16;
}

// Saturation: every codelet input is pre-shifted by log2(r), so |a| <= 2^15 / r
// per component.  Interval analysis of each codelet (tests/test_q15.py::
// test_q15_codelet_intermediates_never_saturate) shows that only the final
// output additions can leave int16; intermediate sums, the sqrdmulh constant
// products and the 32-bit MACs cannot.  Intermediates therefore use plain
// integer arithmetic (identical results); outputs saturate when packed.
// codelet outputs: exact 32-bit sums; the saturation to int16 that sqadd /
// sqsub apply happens when the output is packed (pack_sat)
__device__ __forceinline__ qc qadd(qc a, qc b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ qc qsub(qc a, qc b) { return {a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ qc iadd(qc a, qc b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ qc isub(qc a, qc b) { return {a.re - b.re, a.im - b.im}; }
// sqrdmulh by -32768 is -a for the |a| < 2^15 that reach it
__device__ __forceinline__ qc mul_pi(qc z) { return {-z.im, rdm<32767>(z.re)}; }
__device__ __forceinline__ qc mul_mi(qc z) { return {rdm<32767>(z.im), -z.re}; }
// 32-bit MAC + rounding shift by 15 of in-range operands: the accumulators
// stay far below 2^31 (interval analysis), so adding 2^14 cannot overflow
__device__ __forceinline__ int imac2(int a, int ka, int b, int kb) { return (a * ka + b * kb + 16384) >> 15; }

constexpr int kC8 = 23170, kC16 = 30273, kS16 = 12539;

__device__ __forceinline__ qc mul_w8(qc z) {
  return {imac2(z.re, kC8, rdm<kC8>(z.im), 32767), imac2(z.im, kC8, rdm<kC8>(z.re), -32768)};
}
__device__ __forceinline__ qc mul_w8_3(qc z) {
  return {imac2(z.re, -kC8, rdm<-kC8>(z.im), -32768), imac2(z.im, -kC8, rdm<-kC8>(z.re), 32767)};
}
__device__ __forceinline__ qc mul_w(qc z, int wr, int wi) {
  return {imac2(z.re, wr, z.im, -wi), imac2(z.im, wr, z.re, wi)};
}

// ---- codelets on pre-scaled inputs, outputs in forward order ----
__device__ __forceinline__ void q_dft2(const qc* a, qc* y) {
  y[0] = qadd(a[0], a[1]);
  y[1] = qsub(a[0], a[1]);
}

__device__ __forceinline__ void q_dft4(const qc* a, qc* y) {
  const qc s02 = iadd(a[0], a[2]), s13 = iadd(a[1], a[3]);
  const qc d02 = isub(a[0], a[2]), j13 = mul_pi(isub(a[1], a[3]));
  y[0] = qadd(s02, s13);
  y[2] = qsub(s02, s13);
  y[1] = qsub(d02, j13);
  y[3] = qadd(d02, j13);
}

__device__ __forceinline__ void q_dft8(const qc* a, qc* y) {
  qc p[4], m[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    p[k] = iadd(a[k], a[k + 4]);
    m[k] = isub(a[k], a[k + 4]);
  }
  const qc e0 = iadd(p[0], p[2]), e1 = iadd(p[1], p[3]);
  y[0] = qadd(e0, e1);
  y[4] = qsub(e0, e1);
  const qc d = isub(p[0], p[2]), jd = mul_pi(isub(p[1], p[3]));
  y[2] = qsub(d, jd);
  y[6] = qadd(d, jd);
  const qc z = iadd(m[1], m[3]), w = isub(m[1], m[3]);
  const qc rd = {rdm<kC8>(w.re), rdm<kC8>(w.im)};
  const qc x = {imac2(m[2].im, -32768, z.im, -kC8), imac2(m[2].re, 32767, z.re, kC8)};
  const qc x2 = {imac2(m[2].im, -32768, z.im, kC8), imac2(m[2].re, 32767, z.re, -kC8)};
  const qc u = iadd(m[0], rd), v = isub(m[0], rd);
  y[1] = qsub(u, x);
  y[7] = qadd(u, x);
  y[3] = qadd(v, x2);
  y[5] = qsub(v, x2);
}

__device__ __forceinline__ void q_dft16(const qc* a, qc* y) {
  qc p[8], m[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    p[k] = iadd(a[k], a[k + 8]);
    m[k] = isub(a[k], a[k + 8]);
  }
  const qc s04 = iadd(p[0], p[4]), s26 = iadd(p[2], p[6]);
  const qc s15 = iadd(p[1], p[5]), s37 = iadd(p[3], p[7]);
  const qc e0 = iadd(s04, s26), e1 = iadd(s15, s37);
  y[0] = qadd(e0, e1);
  y[8] = qsub(e0, e1);
  const qc A = isub(s04, s26), jB = mul_pi(isub(s15, s37));
  y[4] = qsub(A, jB);
  y[12] = qadd(A, jB);
  const qc C = isub(p[0], p[4]), jD = mul_pi(isub(p[2], p[6]));
  const qc kE = mul_w8(isub(p[1], p[5])), kF = mul_w8_3(isub(p[3], p[7]));
  const qc g1 = isub(C, jD), g2 = iadd(C, jD);
  const qc h = iadd(kE, kF), h2 = mul_mi(isub(kF, kE));
  y[2] = qadd(g1, h);
  y[10] = qsub(g1, h);
  y[6] = qsub(g2, h2);
  y[14] = qadd(g2, h2);
  const qc j4 = mul_pi(m[4]);
  const qc q = isub(m[0], j4), q2 = iadd(m[0], j4);
  const qc k2 = mul_w8(m[2]), k6 = mul_w8_3(m[6]);
  const qc r = iadd(k2, k6), r2 = mul_mi(isub(k6, k2));
  const qc j5 = mul_pi(m[5]), j7 = mul_pi(m[7]);
  const qc u = isub(m[1], j5), u2 = iadd(m[1], j5);
  const qc v = isub(m[3], j7), v2 = iadd(m[3], j7);
  const qc l1 = mul_w(u, kC16, -kS16), l3 = mul_w(v, kS16, -kC16);
  const qc l3b = mul_w(u2, kS16, -kC16), l9 = mul_w(v2, -kC16, kS16);
  const qc qr = iadd(q, r), qmr = isub(q, r);
  const qc ls = iadd(l1, l3), ld = mul_mi(isub(l3, l1));
  y[1] = qadd(qr, ls);
  y[9] = qsub(qr, ls);
  y[5] = qsub(qmr, ld);
  y[13] = qadd(qmr, ld);
  const qc qa = isub(q2, r2), qb = iadd(q2, r2);
  const qc ls2 = iadd(l3b, l9), ld2 = mul_mi(isub(l9, l3b));
  y[3] = qadd(qa, ls2);
  y[11] = qsub(qa, ls2);
  y[7] = qsub(qb, ld2);
  y[15] = qadd(qb, ld2);
}

template <int R>
__device__ __forceinline__ void q_dft(const qc* a, qc* y) {
  if constexpr (R == 1)
    y[0] = a[0];
  else if constexpr (R == 2)
    q_dft2(a, y);
  else if constexpr (R == 4)
    q_dft4(a, y);
  else if constexpr (R == 8)
    q_dft8(a, y);
  else
    q_dft16(a, y);
}

constexpr int ilog2_c(int r) { return r <= 1 ? 0 : 1 + ilog2_c(r / 2); }

// int16 pair <-> components (little endian: re in the low half)
__device__ __forceinline__ qc unpack(int w) { return {(w << 16) >> 16, w >> 16}; }
// saturate both components to int16 and pack (re in the low half)
__device__ __forceinline__ int pack(qc v) {
  int d;
  asm("cvt.pack.sat.s16.s32 %0, %1, %2;" : "=r"(d) : "r"(v.im), "r"(v.re));
  return d;
}

// n <= 16: one thread per member
template <int N, int DIR>
__global__ void __launch_bounds__(256) q15_small_kernel(const Q15Launch L) {
  griddep_wait();  // launched programmatically (launch_pdl.cuh)
  griddep_launch_dependents();
  const int64_t b = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (b >= L.howmany) return;
  constexpr int S = ilog2_c(N);
  const int* x = L.in + b * L.idist;
  int* y = L.out + b * L.odist;
  qc a[N], r[N];
#pragma unroll
  for (int k = 0; k < N; ++k) {
    const qc v = unpack(x[k * L.istride]);
    a[k] = S ? qc{rshr(v.re, S), rshr(v.im, S)} : v;
  }
  q_dft<N>(a, r);
#pragma unroll
  for (int k = 0; k < N; ++k) y[k * L.ostride] = pack(r[DIR < 0 ? k : (N - k) % N]);
}

// padded shared-memory position of element k (16 columns per row, one
// spare word per row) and the member pitch (== 16 mod 32 words)
__host__ __device__ constexpr int q15_pos(int k) { return k + (k >> 4); }
__host__ __device__ constexpr int q15_pitch(int n) { return ((17 * (n / 16) + 15) / 32) * 32 + 16; }

// n = 16 m, m = 2..16: G = blockDim / 16 members per CTA
template <int N, int DIR>
__global__ void __launch_bounds__(256) q15_two_stage_kernel(const Q15Launch L) {
  griddep_wait();  // launched programmatically (launch_pdl.cuh)
  griddep_launch_dependents();
  constexpr int M = N / 16, SM = ilog2_c(M);
  constexpr int PITCH = q15_pitch(N);
  extern __shared__ int qsm[];
  int2* tw = reinterpret_cast<int2*>(qsm);  // (c, s) and (-s, c) packed pairs
  int* tile = qsm + 2 * 15 * (M - 1 > 0 ? M - 1 : 1);
  const int G = blockDim.x / 16;
  const int64_t b0 = int64_t(blockIdx.x) * G;
  const int64_t left = L.howmany - b0;
  const int cnt = left < G ? int(left) : G;
  for (int i = threadIdx.x; i < 15 * (M - 1); i += blockDim.x) tw[i] = L.tw[i];
  // stage the members (each thread: consecutive elements across members),
  // asynchronous copies so that all of a thread's loads are in flight
  for (int f = threadIdx.x; f < cnt * N; f += blockDim.x) {
    const int g = f / N, k = f - g * N;
    cp_async4(tile + g * PITCH + q15_pos(k), L.in + (b0 + g) * L.idist + int64_t(k) * L.istride);
  }
  cp_async_wait_all();
  __syncthreads();
  const int g = threadIdx.x >> 4, c = threadIdx.x & 15;
  int* mine = tile + g * PITCH;
  if (g < cnt) {  // stage 1: length-M codelet down column c, in place
    qc a[M], r[M];
#pragma unroll
    for (int q = 0; q < M; ++q) {
      const qc v = unpack(mine[q15_pos(c + 16 * q)]);
      a[q] = {rshr(v.re, SM), rshr(v.im, SM)};
    }
    q_dft<M>(a, r);
#pragma unroll
    for (int k = 0; k < M; ++k) mine[q15_pos(c + 16 * k)] = pack(r[DIR < 0 ? k : (M - k) % M]);
  }
  __syncthreads();
  // stage 2: rows (member, j) spread over the CTA's threads
  for (int row = threadIdx.x; row < cnt * M; row += blockDim.x) {
    const int gg = row / M, j = row - gg * M;
    const int* src = tile + gg * PITCH + q15_pos(16 * j);
    qc a[16], r[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const qc v = unpack(src[i]);
      const qc s = {rshr(v.re, 4), rshr(v.im, 4)};
      if (i == 0 || j == 0) {
        a[i] = s;
      } else {
        const int2 w = tw[15 * (j - 1) + (i - 1)];
        const qc cs = unpack(w.x), mc = unpack(w.y);  // (c, s), (-s, c)
        a[i] = {imac2(s.re, cs.re, s.im, mc.re), imac2(s.re, cs.im, s.im, mc.im)};
      }
    }
    q_dft<16>(a, r);
    int* y = L.out + (b0 + gg) * L.odist;
#pragma unroll
    for (int k = 0; k < 16; ++k) y[int64_t(j + M * k) * L.ostride] = pack(r[DIR < 0 ? k : (16 - k) & 15]);
  }
}

bool q15_supported(int64_t n) { return n >= 1 && n <= 256 && (n & (n - 1)) == 0; }

int q15_smem_bytes(int n, int members) {
  if (n <= 16) return 0;
  return 8 * 15 * (n / 16 - 1 > 0 ? n / 16 - 1 : 1) + 4 * members * q15_pitch(n);
}

template <int N, int DIR>
static cudaError_t run_q15(const Q15Launch& L, cudaStream_t st) {
  if constexpr (N <= 16) {
    const int64_t blocks = (L.howmany + 255) / 256;
    return launch_pdl(q15_small_kernel<N, DIR>, dim3(unsigned(blocks)), dim3(256), 0, st, L);
  } else {
    constexpr int kThreads = 256, G = kThreads / 16;
    const int smem = q15_smem_bytes(N, G);
    const int64_t blocks = (L.howmany + G - 1) / G;
    return launch_pdl(q15_two_stage_kernel<N, DIR>, dim3(unsigned(blocks)), dim3(kThreads), size_t(smem), st, L);
  }
}

cudaError_t launch_q15(int n, int dir, const Q15Launch& L, cudaStream_t st) {
#define PLFFT_B200_Q15(NV) \
  if (n == NV) return dir < 0 ? run_q15<NV, -1>(L, st) : run_q15<NV, 1>(L, st);
  PLFFT_B200_Q15(1)
  PLFFT_B200_Q15(2)
  PLFFT_B200_Q15(4)
  PLFFT_B200_Q15(8)
  PLFFT_B200_Q15(16)
  PLFFT_B200_Q15(32)
  PLFFT_B200_Q15(64)
  PLFFT_B200_Q15(128)
  PLFFT_B200_Q15(256)
#undef PLFFT_B200_Q15
  return cudaErrorInvalidValue;
}

}  // namespace plfft_b200
