// Batched complex-to-complex FP32 kernels.
//
// c2c_reg_kernel : register engine, one transform per T = n/E threads,
//                  G transforms per CTA; the batch-member loop of the
//                  reference (src/batched_1d_plan.hpp:85-128 and the
//                  planner's loop strategy, src/planner/strategies/loop.hpp:
//                  29-35) becomes the grid.
// c2c_tile_kernel: shared-memory engine over a tile of C transforms with
//                  arbitrary element/transform strides; load and store each
//                  walk the contiguous dimension so both stay coalesced.
//                  Also serves as a four-step pass (optional twiddle on the
//                  outputs), the role of the reference's twiddled Cooley-Tukey
//                  levels (src/level_ac_t_c2c.cpp:50-85,
//                  src/level_ab_t_c2c.cpp:49-80).
#include "kernels.h"
#include "stockham.cuh"
#include "ptx.cuh"

namespace plfft_b200 {

template <int E, int DIR>
__global__ void __launch_bounds__(256) c2c_reg_kernel(const RegLaunch L) {
  extern __shared__ float2 smem[];
  const int T = L.t;
  const int grp = threadIdx.x / T;
  const int t = threadIdx.x - grp * T;
  const int64_t b = int64_t(blockIdx.x) * L.g + grp;
  const bool live = b < L.howmany;
  float2* sm = smem + grp * spad_len(L.desc.n);

  float2 v[E];
  if (live) {
    const float2* src = L.in + b * L.idist;
#pragma unroll
    for (int q = 0; q < E; ++q) v[q] = src[int64_t(t + T * q) * L.istride];
  } else {
#pragma unroll
    for (int q = 0; q < E; ++q) v[q] = make_float2(0.f, 0.f);
  }
  const GroupSync sync{!(T <= 32 && (32 % T) == 0)};
  reg_fft<E, DIR>(v, L.desc, t, T, sm, L.tw, sync);
  if (live) {
    float2* dst = L.out + b * L.odist;
    const float s = L.scale;
#pragma unroll
    for (int q = 0; q < E; ++q) dst[int64_t(t + T * q) * L.ostride] = s == 1.f ? v[q] : cscale(v[q], s);
  }
}

__device__ __forceinline__ int64_t tile_base(const Addr& a, int64_t g) {
  const int64_t m = g / a.ncols;
  const int64_t c = g - m * a.ncols;
  return m * a.mdist + c * a.cdist;
}

// W_N^e for 0 <= e < N from two short tables: lo[e % L] * hi[e / L]
__device__ __forceinline__ float2 two_level(const TwoLevel& p, int e) {
  const int hi = e / p.l;
  const int lo = e - hi * p.l;
  return cmul(__ldg(p.lo + lo), __ldg(p.hi + hi));
}

// per-thread element budget -> largest CTA that keeps it in registers
#define PLFFT_B200_TILE_THREADS(MAXE) ((MAXE) <= 16 ? 512 : 256)

constexpr int kMaxTileC = 64;

// two resident CTAs of the largest size: caps registers at 64 (16
// elements per thread) or 128 (32) with no spills, so a typical 288-thread
// tile fits three CTAs per SM instead of two
template <int MAXE, int DIR>
__global__ void __launch_bounds__(PLFFT_B200_TILE_THREADS(MAXE), 2) c2c_tile_kernel(const TileLaunch L) {
  extern __shared__ float2 smem[];
  __shared__ int64_t ibase[kMaxTileC], obase[kMaxTileC];
  __shared__ int colidx[kMaxTileC];
  const int n = L.desc.n;
  const int C = L.c;
  const int ld = L.ld;
  const int tid = threadIdx.x;
  const int nthr = blockDim.x;
  const int64_t g0 = int64_t(blockIdx.x) * C;
  const int64_t rem = L.ntr - g0;
  const int cnt = rem < C ? int(rem) : C;
  const int total = cnt * n;
  if (tid < cnt) {
    ibase[tid] = tile_base(L.ia, g0 + tid);
    obase[tid] = tile_base(L.oa, g0 + tid);
    colidx[tid] = int((g0 + tid) % L.ia.ncols);
  }
  __syncthreads();

  // load: walk k fastest when elements are contiguous, else walk c fastest
  const int64_t iks = L.ia.kstride;
  if (iks == 1) {
    for (int f = tid; f < total; f += nthr) {
      const int c = f / n, k = f - c * n;
      cp_async8(smem + c * ld + spad(k), L.in + ibase[c] + k);
    }
  } else {
    for (int f = tid; f < total; f += nthr) {
      const int k = f / cnt, c = f - k * cnt;
      cp_async8(smem + c * ld + spad(k), L.in + ibase[c] + k * iks);
    }
  }
  cp_async_wait_all();
  __syncthreads();
  smem_fft<MAXE, DIR>(smem, cnt, ld, L.desc, L.tw, tid, nthr);

  const float s = L.scale;
  const int64_t oks = L.oa.kstride;
  const bool post = L.post.n != 0;
  if (oks == 1) {
    for (int f = tid; f < total; f += nthr) {
      const int c = f / n, k = f - c * n;
      float2 y = smem[c * ld + spad(k)];
      if (post) y = twmul<DIR>(y, two_level(L.post, colidx[c] * k));
      if (s != 1.f) y = cscale(y, s);
      L.out[obase[c] + k] = y;
    }
  } else {
    for (int f = tid; f < total; f += nthr) {
      const int k = f / cnt, c = f - k * cnt;
      float2 y = smem[c * ld + spad(k)];
      if (post) y = twmul<DIR>(y, two_level(L.post, colidx[c] * k));
      if (s != 1.f) y = cscale(y, s);
      L.out[obase[c] + k * oks] = y;
    }
  }
}

int reg_smem_bytes(int n, int g) { return g * spad_len(n) * int(sizeof(float2)); }
int tile_smem_bytes(int ld, int c) { return ld * c * int(sizeof(float2)); }

template <class K>
static cudaError_t set_smem(K kernel, int bytes) {
  return ensure_dynamic_smem(reinterpret_cast<const void*>(kernel), bytes);
}

template <int E, int DIR>
static cudaError_t run_reg(const RegLaunch& L, cudaStream_t st) {
  const int smem = reg_smem_bytes(L.desc.n, L.g);
  cudaError_t e = set_smem(c2c_reg_kernel<E, DIR>, smem);
  if (e != cudaSuccess) return e;
  const int64_t blocks = (L.howmany + L.g - 1) / L.g;
  c2c_reg_kernel<E, DIR><<<dim3(unsigned(blocks)), dim3(L.t * L.g), smem, st>>>(L);
  return cudaGetLastError();
}

cudaError_t launch_c2c_reg(int e, int dir, const RegLaunch& L, cudaStream_t st) {
#define PLFFT_B200_E(EV)                                                  \
  if (e == EV) return dir < 0 ? run_reg<EV, -1>(L, st) : run_reg<EV, 1>(L, st);
  PLFFT_B200_E(2)
  PLFFT_B200_E(4)
  PLFFT_B200_E(8)
  PLFFT_B200_E(16)
  PLFFT_B200_E(32)
#undef PLFFT_B200_E
  return cudaErrorInvalidValue;
}

template <int MAXE, int DIR>
static cudaError_t run_tile(const TileLaunch& L, cudaStream_t st) {
  const int smem = tile_smem_bytes(L.ld, L.c);
  cudaError_t e = set_smem(c2c_tile_kernel<MAXE, DIR>, smem);
  if (e != cudaSuccess) return e;
  const int64_t blocks = (L.ntr + L.c - 1) / L.c;
  c2c_tile_kernel<MAXE, DIR><<<dim3(unsigned(blocks)), dim3(L.nthr), smem, st>>>(L);
  return cudaGetLastError();
}

cudaError_t launch_c2c_tile(int maxe, int dir, const TileLaunch& L, cudaStream_t st) {
  if (maxe == 16) return dir < 0 ? run_tile<16, -1>(L, st) : run_tile<16, 1>(L, st);
  if (maxe == 32) return dir < 0 ? run_tile<32, -1>(L, st) : run_tile<32, 1>(L, st);
  return cudaErrorInvalidValue;
}

}  // namespace plfft_b200
