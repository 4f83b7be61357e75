// Persistent grouped kernel: thousands of C2C FP32 transforms of mixed
// length in one launch per dependency phase.
//
// A group (grouped_plan.cpp) is a list of tasks.  Every task is one of:
//   GT_TILE   : `cnt` transforms (or four-step columns/rows) of one on-chip
//               length, element (c, k) at base + c*cdist + k*kstride, with an
//               optional prologue op on the loaded values and an optional
//               epilogue op on the results;
//   GT_RADER  : a whole Rader transform of prime length P, P-1 on chip;
//   GT_BLUE   : a whole Bluestein transform whose length-M convolution fits
//               on chip.
// Lengths that do not fit on chip become four-step tiles in two phases (and
// Rader/Bluestein convolutions of such lengths in four).  CTAs are resident
// for the whole phase and take tasks from a device counter in order of
// decreasing cost; the last CTA to finish resets the counter, so a captured
// CUDA graph can be replayed.
//
// This replaces, for mixed batches, the one-plan-per-length execution a
// PLFFT user would otherwise run (a plan per length, reference
// src/plfft.cpp:427-517 and the batched plan of src/batched_1d_plan.hpp).
#include "kernels.h"
#include "ptx.cuh"
#include "stockham.cuh"

namespace plfft_b200 {

constexpr int kGroupMaxE = 32;
constexpr int kGroupThreads = 256;

__device__ __forceinline__ float2 group_two_level(const TwoLevel& p, int64_t e) {
  e %= p.n;
  const int64_t hi = e / p.l;
  const int64_t lo = e - hi * p.l;
  return cmul(__ldg(p.lo + lo), __ldg(p.hi + hi));
}

template <int DIR>
__device__ __forceinline__ void group_fft(float2* sm, int cnt, int ld, const GroupPhase& P, int desc) {
  smem_fft<kGroupMaxE, DIR>(sm, cnt, ld, P.descs[desc], P.tws[desc], threadIdx.x, blockDim.x);
}

__device__ __forceinline__ void group_fft_dir(int dir, float2* sm, int cnt, int ld, const GroupPhase& P, int desc) {
  if (dir < 0)
    group_fft<-1>(sm, cnt, ld, P, desc);
  else
    group_fft<1>(sm, cnt, ld, P, desc);
}

// epilogue: store result element (c, k) of a tile
__device__ __forceinline__ void tile_store(const GTask& T, float2* out, const float2* xin, int c, int k, float2 y,
                                           int dir) {
  const int64_t e = T.oe0 + int64_t(c) * T.oec + int64_t(k) * T.oek;  // logical output index
  switch (T.post_op) {
    case GO_TWIDDLE: {
      const float2 w = group_two_level(T.tw2, (T.col0 + c) * int64_t(k));
      y = dir < 0 ? cmul(y, w) : cmulc(y, w);
      break;
    }
    case GO_SPEC:
      y = cmul(y, T.post_tab[e]);
      break;
    case GO_SPEC_SAVE0:
      if (e == 0) T.sum0[0] = y;
      y = cmul(y, T.post_tab[e]);
      break;
    case GO_CHIRP:
      if (e >= T.post_len) return;
      y = cmul(y, T.post_tab[e]);
      break;
    case GO_SCATTER: {
      const float2 x0 = xin[0];
      out[int64_t(T.perm_out[e]) * T.okstride] = cscale(cadd(x0, y), T.scale);
      if (e == 0) out[0] = cscale(cadd(x0, T.sum0[0]), T.scale);
      return;
    }
    default:
      break;
  }
  out[int64_t(c) * T.ocdist + int64_t(k) * T.okstride] = T.scale == 1.f ? y : cscale(y, T.scale);
}

__device__ void run_tile(const GTask& T, const GroupPhase& P, float2* sm) {
  const int n = T.n, cnt = T.cnt;
  const int ld = spad_len(n);
  const int total = cnt * n;
  const float2* in = P.bases[T.in_buf] + T.in_off;
  float2* out = P.bases[T.out_buf] + T.out_off;
  const float2* xin = P.bases[T.aux_buf] + T.aux_off;
  // element f = (c, k) walks the tile with the fast index along the
  // contiguous dimension; (c, k) is carried from one iteration to the next
  // (one division per tile, not per element) and the loop is unrolled so
  // that several loads are in flight per thread
  const bool kfast_in = T.ikstride == 1 || T.pre_op == GO_GATHER;
  {
    const int fast = kfast_in ? n : cnt;  // extent of the fast index
    const int bq = blockDim.x / fast, br = blockDim.x - bq * fast;
    int slow = threadIdx.x / fast, fi = threadIdx.x - slow * fast;
    // asynchronous copies (all of a thread's loads in flight); the chirp of
    // a Bluestein prologue is applied in shared memory afterwards
#pragma unroll 4
    for (int f = threadIdx.x; f < total; f += blockDim.x) {
      const int c = kfast_in ? slow : fi, k = kfast_in ? fi : slow;
      float2* dst = sm + c * ld + spad(k);
      if (T.pre_op == GO_GATHER) {
        const int64_t e = T.ie0 + int64_t(c) * T.iec + int64_t(k) * T.iek;
        cp_async8(dst, in + int64_t(T.perm_in[e]) * T.ikstride);
      } else if (T.pre_op == GO_CHIRP && T.ie0 + int64_t(c) * T.iec + int64_t(k) * T.iek >= T.pre_len) {
        *dst = make_float2(0.f, 0.f);
      } else {
        cp_async8(dst, in + int64_t(c) * T.icdist + int64_t(k) * T.ikstride);
      }
      fi += br;
      slow += bq;
      if (fi >= fast) {
        fi -= fast;
        ++slow;
      }
    }
    cp_async_wait_all();
    if (T.pre_op == GO_CHIRP) {
      __syncthreads();
      for (int f = threadIdx.x; f < total; f += blockDim.x) {
        const int c = f / n, k = f - c * n;
        const int64_t e = T.ie0 + int64_t(c) * T.iec + int64_t(k) * T.iek;
        if (e < T.pre_len) sm[c * ld + spad(k)] = cmul(sm[c * ld + spad(k)], T.pre_tab[e]);
      }
    }
  }
  __syncthreads();
  group_fft_dir(T.dir, sm, cnt, ld, P, T.desc);
  const bool kfast_out = T.okstride == 1 || T.post_op == GO_SCATTER;
  {
    const int fast = kfast_out ? n : cnt;
    const int bq = blockDim.x / fast, br = blockDim.x - bq * fast;
    int slow = threadIdx.x / fast, fi = threadIdx.x - slow * fast;
#pragma unroll 4
    for (int f = threadIdx.x; f < total; f += blockDim.x) {
      const int c = kfast_out ? slow : fi, k = kfast_out ? fi : slow;
      tile_store(T, out, xin, c, k, sm[c * ld + spad(k)], T.dir);
      fi += br;
      slow += bq;
      if (fi >= fast) {
        fi -= fast;
        ++slow;
      }
    }
  }
}

// whole Rader transform (P prime, P-1 = T.n on chip)
__device__ void run_rader(const GTask& T, const GroupPhase& P, float2* sm) {
  const int m = T.n;
  const int ld = spad_len(m);
  const float2* in = P.bases[T.in_buf] + T.in_off;
  float2* out = P.bases[T.out_buf] + T.out_off;
  __shared__ float2 a0;
  for (int q = threadIdx.x; q < m; q += blockDim.x) sm[spad(q)] = in[int64_t(T.perm_in[q]) * T.ikstride];
  __syncthreads();
  group_fft<-1>(sm, 1, ld, P, T.desc);
  if (threadIdx.x == 0) a0 = sm[0];
  __syncthreads();
  for (int q = threadIdx.x; q < m; q += blockDim.x) sm[spad(q)] = cmul(sm[spad(q)], T.post_tab[q]);
  __syncthreads();
  group_fft<1>(sm, 1, ld, P, T.desc);
  const float2 x0 = in[0];
  for (int q = threadIdx.x; q < m; q += blockDim.x)
    out[int64_t(T.perm_out[q]) * T.okstride] = cscale(cadd(x0, sm[spad(q)]), T.scale);
  if (threadIdx.x == 0) out[0] = cscale(cadd(x0, a0), T.scale);
}

// whole Bluestein transform (length T.pre_len, convolution length T.n on chip)
__device__ void run_blue(const GTask& T, const GroupPhase& P, float2* sm) {
  const int m = T.n, nl = T.pre_len;
  const int ld = spad_len(m);
  const float2* in = P.bases[T.in_buf] + T.in_off;
  float2* out = P.bases[T.out_buf] + T.out_off;
  for (int j = threadIdx.x; j < m; j += blockDim.x)
    sm[spad(j)] = j < nl ? cmul(in[int64_t(j) * T.ikstride], T.pre_tab[j]) : make_float2(0.f, 0.f);
  __syncthreads();
  group_fft<-1>(sm, 1, ld, P, T.desc);
  for (int k = threadIdx.x; k < m; k += blockDim.x) sm[spad(k)] = cmul(sm[spad(k)], T.post_tab2[k]);
  __syncthreads();
  group_fft<1>(sm, 1, ld, P, T.desc);
  for (int k = threadIdx.x; k < nl; k += blockDim.x)
    out[int64_t(k) * T.okstride] = cscale(cmul(sm[spad(k)], T.pre_tab[k]), T.scale);
}

__global__ void __launch_bounds__(kGroupThreads, 2) grouped_kernel(const GroupPhase P) {
  extern __shared__ float2 smem[];
  __shared__ int cur;
  for (;;) {
    if (threadIdx.x == 0) cur = atomicAdd(P.counter, 1);
    __syncthreads();
    const int t = cur;
    __syncthreads();
    if (t >= P.ntasks) break;
    const GTask T = P.tasks[t];
    switch (T.type) {
      case GT_TILE: run_tile(T, P, smem); break;
      case GT_RADER: run_rader(T, P, smem); break;
      case GT_BLUE: run_blue(T, P, smem); break;
      default: break;
    }
    __syncthreads();
  }
  // the last CTA out resets the counters for the next launch / graph replay
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(P.done, 1) == int(gridDim.x) - 1) {
      *P.counter = 0;
      *P.done = 0;
      __threadfence();
    }
  }
}

int group_max_smem_elems() { return 72 * 1024 / int(sizeof(float2)); }

cudaError_t launch_grouped(const GroupPhase& P, int grid, int smem_bytes, cudaStream_t st) {
  cudaError_t e = cudaFuncSetAttribute(grouped_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes);
  if (e != cudaSuccess) return e;
  grouped_kernel<<<grid, kGroupThreads, smem_bytes, st>>>(P);
  return cudaGetLastError();
}

int grouped_blocks_per_sm(int smem_bytes) {
  int per = 0;
  cudaFuncSetAttribute(grouped_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, grouped_kernel, kGroupThreads, smem_bytes);
  return per < 1 ? 1 : per;
}

}  // namespace plfft_b200
