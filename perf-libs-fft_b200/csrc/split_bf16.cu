// Split-BF16 tensor-core C2C pass: on-chip FFTs of length NL = 16^s whose
// radix-16 stages are DFT-matrix products on the tensor cores.
//
// Precision scheme: every FP32 operand is split into three BF16 terms,
// x = x0 + x1 + x2 (x0 = bf16(x), x1 = bf16(x - x0), x2 = bf16(x - x0 - x1)),
// which carries the full 24-bit significand.  The radix-16 DFT matrix
// (as the real 32x32 matrix [Re W, -Im W; Im W, Re W], computed in FP64 on
// the host) is split the same way.  A stage accumulates the six cross
// products with i + j <= 2 (W2 x0, W1 x1, W0 x2, W1 x0, W0 x1, W0 x0, small
// terms first) in FP32 inside the tensor core; the dropped terms are below
// 2^-24 relative.  Twiddles between stages and the four-step twiddle are
// applied in FP32 on the CUDA cores.  The reference has no counterpart; its
// nearest analogue is the SME2 DFT-matrix outer-product kernel
// (src/planner/strategies/direct_sme2.hpp:27-95).
//
// Data flow of one CTA: a tile of C = 4096 / NL sub-transforms is loaded
// into shared memory (padded positions p + p/16), then for each Stockham
// stage (Ns = 16^t) every column v = (sub-transform, j) forms the 16-vector
// u_q = x[j + q NL/16] * W_{16 Ns}^{(j mod Ns) q}; eight columns make one
// m16n8k16 B operand per real/imaginary half; the outputs y_i go to
// x'[(j / Ns) 16 Ns + j mod Ns + i Ns].  After the last stage the tile is
// in natural order; the store applies the four-step twiddle and scale.
#include <cuda_bf16.h>

#include "kernels.h"
#include "ptx.cuh"
#include "stockham.cuh"

namespace plfft_b200 {

constexpr int kSbThreads = 256;
constexpr int kSbTile = 4096;  // complex elements per CTA tile


// three-term split of a pair of floats into packed bf16x2 words by
// truncation: the high 16 bits of a float are a bf16 value, so
// x0 = hi16(x), r = x - x0 (exact), x1 = hi16(r), r2 = r - x1 (exact),
// x2 = hi16(r2); the three 8-bit significands carry 24 bits of x, and
// __byte_perm gathers the high halves of two floats into one word
__device__ __forceinline__ float hi16(float x) { return __uint_as_float(__float_as_uint(x) & 0xffff0000u); }
__device__ __forceinline__ uint32_t pack_hi(float lo, float hi) {
  return __byte_perm(__float_as_uint(lo), __float_as_uint(hi), 0x7632);
}
__device__ __forceinline__ void split3(float a, float b, uint32_t& w0, uint32_t& w1, uint32_t& w2) {
  const float ra = a - hi16(a), rb = b - hi16(b);
  const float r2a = ra - hi16(ra), r2b = rb - hi16(rb);
  w0 = pack_hi(a, b);
  w1 = pack_hi(ra, rb);
  w2 = pack_hi(r2a, r2b);
}

// D += A (16x16 bf16, row) * B (16x8 bf16, col), FP32 accumulate (no side
// effects, so not volatile: the compiler may interleave independent MMAs)
__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// W_n^e = lo[e mod L] * hi[e / L]
__device__ __forceinline__ float2 sb_two_level(const TwoLevel& p, uint32_t e, int lshift) {
  return cmul(__ldg(p.lo + (e & uint32_t(p.l - 1))), __ldg(p.hi + (e >> lshift)));
}

// A-operand fragments of the split 32x32 real DFT-16 matrix: [split][m-tile][k-step][4]
struct SbA {
  uint32_t r[3][2][2][4];
};

// mat: three 32x32 row-major bf16 matrices (bf16 pairs as 32-bit words)
__device__ __forceinline__ void load_a(SbA& A, const uint32_t* __restrict__ mat, int g, int t) {
#pragma unroll
  for (int s = 0; s < 3; ++s)
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
      for (int ks = 0; ks < 2; ++ks) {
        const uint32_t* m = mat + s * 512;  // 32 rows x 16 words
        const int r0 = mt * 16 + g, c0 = ks * 8 + t;  // word column = (ks*16 + 2t)/2
        A.r[s][mt][ks][0] = __ldg(m + r0 * 16 + c0);
        A.r[s][mt][ks][1] = __ldg(m + (r0 + 8) * 16 + c0);
        A.r[s][mt][ks][2] = __ldg(m + r0 * 16 + c0 + 4);
        A.r[s][mt][ks][3] = __ldg(m + (r0 + 8) * 16 + c0 + 4);
      }
}

// One radix-16 Stockham stage over the tile: V = C * NL / 16 columns, each
// warp takes n-tiles of 8 columns.  Outputs are written after a barrier so
// the stage runs in place.
template <int NL, int DIR, int NT>
__device__ __forceinline__ void sb_stage(float2* tile, int pitch, int ns, const float2* __restrict__ tw,
                                         const SbA& A, int warp, int g, int t) {
  constexpr int J = NL / 16;  // columns per sub-transform
  float acc[NT][2][4];
  // n-tiles in pairs: the two tiles' MMAs alternate, so consecutive MMAs
  // accumulate into different registers
#pragma unroll
  for (int it0 = 0; it0 < NT; it0 += 2) {
    uint32_t b[2][3][2][2];  // [tile][split][k-step][reg]
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      const int v = (warp * NT + it0 + p) * 8 + g;  // this thread's B column
      const int c = v / J, j = v - c * J;
      const float2* x = tile + c * pitch;
      const int r = j & (ns - 1);
      // u_q for q in {2t, 2t+1, 2t+8, 2t+9}, twiddled by W_{16 ns}^{r q}
      float2 u[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int q = 2 * t + (e & 1) + (e >> 1) * 8;
        float2 val = x[spad(j + q * J)];
        if (ns > 1 && q > 0) val = twmul<DIR>(val, tw[(q - 1) * ns + r]);
        u[e] = val;
      }
      // B operands: k-step 0 = real parts, k-step 1 = imaginary parts
      split3(u[0].x, u[1].x, b[p][0][0][0], b[p][1][0][0], b[p][2][0][0]);
      split3(u[2].x, u[3].x, b[p][0][0][1], b[p][1][0][1], b[p][2][0][1]);
      split3(u[0].y, u[1].y, b[p][0][1][0], b[p][1][1][0], b[p][2][1][0]);
      split3(u[2].y, u[3].y, b[p][0][1][1], b[p][1][1][1], b[p][2][1][1]);
#pragma unroll
      for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int i = 0; i < 4; ++i) acc[it0 + p][mt][i] = 0.f;
    }
    // products W_sa x_sb with sa + sb <= 2, smallest first
    constexpr int kSa[6] = {2, 1, 0, 1, 0, 0};
    constexpr int kSb[6] = {0, 1, 2, 0, 1, 0};
#pragma unroll
    for (int term = 0; term < 6; ++term)
#pragma unroll
      for (int ks = 0; ks < 2; ++ks)
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
          for (int p = 0; p < 2; ++p)
            mma_bf16(acc[it0 + p][mt], A.r[kSa[term]][mt][ks], b[p][kSb[term]][ks][0], b[p][kSb[term]][ks][1]);
  }
  __syncthreads();  // every column of this stage has been read
#pragma unroll
  for (int it = 0; it < NT; ++it) {
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int v = (warp * NT + it) * 8 + 2 * t + e;  // C-fragment columns 2t, 2t+1
      const int c = v / J, j = v - c * J;
      float2* y = tile + c * pitch;
      const int base = (j & ~(ns - 1)) * 16 + (j & (ns - 1));
      // rows g and g + 8 of the real (m-tile 0) and imaginary (m-tile 1) halves
      y[spad(base + g * ns)] = make_float2(acc[it][0][e], acc[it][1][e]);
      y[spad(base + (g + 8) * ns)] = make_float2(acc[it][0][2 + e], acc[it][1][2 + e]);
    }
  }
  __syncthreads();
}

template <int NL, int DIR>
__global__ void __launch_bounds__(kSbThreads, 2) split_bf16_pass_kernel(const FourStepLaunch L,
                                                                     const uint32_t* __restrict__ dftm) {
  constexpr int C = kSbTile / NL;  // sub-transforms per CTA
  constexpr int S = NL == 256 ? 2 : 3;
  constexpr int PITCH = (spad_len_c(NL) + 1) & ~1;
  constexpr int NT = kSbTile / 16 / 8 / (kSbThreads / 32);  // n-tiles per warp and stage
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ int64_t ibase[C], obase[C], colv[C];
  float2* tile = reinterpret_cast<float2*>(smraw);
  const int64_t g0 = int64_t(blockIdx.x) * C;
  const int64_t rem = L.count - g0;
  const int cnt = rem < C ? int(rem) : C;
  if (threadIdx.x < cnt) {
    const int64_t gi = g0 + threadIdx.x;
    const int64_t m = gi / L.ncols;
    const int64_t col = gi - m * L.ncols;
    ibase[threadIdx.x] = m * L.imdist + col * L.icd;
    obase[threadIdx.x] = m * L.omdist + col * L.ocd;
    colv[threadIdx.x] = col;
  }
  __syncthreads();
  const int total = cnt * NL;
  if (L.iks == 1) {
    for (int f = threadIdx.x; f < total; f += blockDim.x) {
      const int c = f / NL, k = f - c * NL;
      cp_async8(tile + c * PITCH + spad(k), L.in + ibase[c] + k);
    }
  } else {
    for (int f = threadIdx.x; f < total; f += blockDim.x) {
      const int k = f / cnt, c = f - k * cnt;
      cp_async8(tile + c * PITCH + spad(k), L.in + ibase[c] + int64_t(k) * L.iks);
    }
  }
  // members past the batch end: zeros, so every column of the tile is defined
  for (int f = total + threadIdx.x; f < C * NL; f += blockDim.x) {
    const int c = f / NL, k = f - c * NL;
    tile[c * PITCH + spad(k)] = make_float2(0.f, 0.f);
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  SbA A;
  load_a(A, dftm, g, t);
  cp_async_wait_all();
  __syncthreads();
  int ns = 1, twoff = 0;
#pragma unroll 1
  for (int s = 0; s < S; ++s) {
    sb_stage<NL, DIR, NT>(tile, PITCH, ns, L.tw + twoff, A, warp, g, t);
    if (s >= 1) twoff += 15 * ns;
    ns *= 16;
  }
  const bool post = L.post.n != 0;
  const int lshift = __ffs(L.post.l) - 1;
  if (L.oks == 1) {
    for (int f = threadIdx.x; f < total; f += blockDim.x) {
      const int c = f / NL, k = f - c * NL;
      float2 v = tile[c * PITCH + spad(k)];
      if (post) v = twmul<DIR>(v, sb_two_level(L.post, uint32_t(colv[c]) * uint32_t(k), lshift));
      L.out[obase[c] + k] = cscale(v, L.scale);
    }
  } else {
    for (int f = threadIdx.x; f < total; f += blockDim.x) {
      const int k = f / cnt, c = f - k * cnt;
      float2 v = tile[c * PITCH + spad(k)];
      if (post) v = twmul<DIR>(v, sb_two_level(L.post, uint32_t(colv[c]) * uint32_t(k), lshift));
      L.out[obase[c] + int64_t(k) * L.oks] = cscale(v, L.scale);
    }
  }
}

bool split_bf16_pass_supported(int nl) { return nl == 256 || nl == 4096; }

int split_bf16_pass_c(int nl) { return kSbTile / nl; }

template <int NL, int DIR>
static cudaError_t run_sb(const FourStepLaunch& L, const uint32_t* dftm, cudaStream_t st) {
  constexpr int C = kSbTile / NL;
  const int smem = C * ((spad_len(NL) + 1) & ~1) * int(sizeof(float2));
  {
    const cudaError_t e = ensure_dynamic_smem(reinterpret_cast<const void*>(split_bf16_pass_kernel<NL, DIR>), smem);
    if (e != cudaSuccess) return e;
  }
  const int64_t blocks = (L.count + C - 1) / C;
  split_bf16_pass_kernel<NL, DIR><<<dim3(unsigned(blocks)), dim3(kSbThreads), smem, st>>>(L, dftm);
  return cudaGetLastError();
}

cudaError_t launch_split_bf16_pass(int nl, int dir, const FourStepLaunch& L, const uint32_t* dftm,
                                   cudaStream_t st) {
  if (nl == 256) return dir < 0 ? run_sb<256, -1>(L, dftm, st) : run_sb<256, 1>(L, dftm, st);
  if (nl == 4096) return dir < 0 ? run_sb<4096, -1>(L, dftm, st) : run_sb<4096, 1>(L, dftm, st);
  return cudaErrorInvalidValue;
}

}  // namespace plfft_b200
