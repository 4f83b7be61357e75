// Power-of-two four-step passes with compile-time stage lists.
//
// A transform of length n = n1 * n2 runs as two passes (the reference's
// twiddled Cooley-Tukey levels, src/level_ac_t_c2c.cpp:50-85 and
// src/level_ab_t_c2c.cpp:49-80, with one on-chip FFT per pass):
//   pass 1: n2 column FFTs of length n1 over stride n2, outputs times
//           W_n^{column * k1}, written back in the same layout;
//   pass 2: n1 row FFTs of length n2 (contiguous), written transposed to
//           X[k1 + n1 k2].
// A CTA takes C sub-transforms.  The tile is loaded into per-sub-transform
// shared-memory slots walking the contiguous dimension (columns: C adjacent
// elements per row; rows: along the row), each slot is transformed by its
// group of T = nl/E threads in registers, and the tile is stored walking the
// contiguous dimension of the output.
#include "kernels.h"
#include "launch_pdl.cuh"
#include "pow2_stages.cuh"
#include "ptx.cuh"

namespace plfft_b200 {

constexpr int kFourStepMaxC = 32;

// W_n^e = lo[e mod L] * hi[e / L]; e < n <= 2^31 and L is a power of two
__device__ __forceinline__ float2 fs_two_level(const TwoLevel& p, uint32_t e, int lshift) {
  return cmul(__ldg(p.lo + (e & uint32_t(p.l - 1))), __ldg(p.hi + (e >> lshift)));
}

template <int NL, int E, int DIR>
__global__ void __launch_bounds__(512) fourstep_pass_kernel(const FourStepLaunch L) {
  griddep_wait();  // launched programmatically (launch_pdl.cuh)
  griddep_launch_dependents();
  using P = P2<NL, E>;
  constexpr int T = P::T;
  constexpr int PITCH = (spad_len_c(NL) + 1) & ~1;
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ int64_t ibase[kFourStepMaxC], obase[kFourStepMaxC], colv[kFourStepMaxC];
  float2* slots = reinterpret_cast<float2*>(smraw);
  const int C = L.c;
  const int grp = threadIdx.x / T;
  const int t = threadIdx.x - grp * T;
  const int64_t g0 = int64_t(blockIdx.x) * C;
  const int64_t rem = L.count - g0;
  const int cnt = rem < C ? int(rem) : C;
  if (threadIdx.x < cnt) {
    const int64_t g = g0 + threadIdx.x;
    const int64_t m = g / L.ncols;
    const int64_t col = g - m * L.ncols;
    ibase[threadIdx.x] = m * L.imdist + col * L.icd;
    obase[threadIdx.x] = m * L.omdist + col * L.ocd;
    colv[threadIdx.x] = col;
  }
  __syncthreads();
  const int total = cnt * NL;
  if (L.iks == 1) {
    for (int f = threadIdx.x; f < total; f += blockDim.x) {
      const int c = f / NL, k = f - c * NL;
      cp_async8(slots + c * PITCH + k, L.in + ibase[c] + k);
    }
  } else if ((cnt & (cnt - 1)) == 0) {  // full power-of-two tile: shifts, no division
    const int sh = __ffs(cnt) - 1;
    for (int f = threadIdx.x; f < total; f += blockDim.x) {
      const int k = f >> sh, c = f & (cnt - 1);
      cp_async8(slots + c * PITCH + k, L.in + ibase[c] + int64_t(k) * L.iks);
    }
  } else {
    for (int f = threadIdx.x; f < total; f += blockDim.x) {
      const int k = f / cnt, c = f - k * cnt;
      cp_async8(slots + c * PITCH + k, L.in + ibase[c] + int64_t(k) * L.iks);
    }
  }
  cp_async_wait_all();
  __syncthreads();
  float2* mine = slots + grp * PITCH;
  auto sync = [&]() {
    if constexpr (T <= 32)
      __syncwarp();
    else
      __syncthreads();
  };
  float2 v[E];
#pragma unroll
  for (int q = 0; q < E; ++q) v[q] = mine[t + T * q];
  st_bfly<T, E, P::radix(0), 1, 0, DIR>(v, t, L.tw);
  Stages<NL, E, DIR, 1>::run(v, t, mine, L.tw, sync);
  if (L.post.n != 0 && grp < cnt) {
    // W_n^{col k}, k = t + T q: a table lookup every fourth q and a product
    // with W_n^{col T} in between (at most three extra roundings, a quarter
    // of the table loads)
    const uint32_t col = uint32_t(colv[grp]);
    const int lshift = __ffs(L.post.l) - 1;
    const float2 step = fs_two_level(L.post, col * uint32_t(T), lshift);
    float2 w = make_float2(1.f, 0.f);
#pragma unroll
    for (int q = 0; q < E; ++q) {
      w = (q & 3) == 0 ? fs_two_level(L.post, col * uint32_t(t + T * q), lshift) : cmul(w, step);
      v[q] = twmul<DIR>(v[q], w);
    }
  }
  if (L.scale != 1.f) {
#pragma unroll
    for (int q = 0; q < E; ++q) v[q] = cscale(v[q], L.scale);
  }
  sync();
#pragma unroll
  for (int q = 0; q < E; ++q) mine[t + T * q] = v[q];
  __syncthreads();
  if (L.oks == 1) {
    for (int f = threadIdx.x; f < total; f += blockDim.x) {
      const int c = f / NL, k = f - c * NL;
      L.out[obase[c] + k] = slots[c * PITCH + k];
    }
  } else if ((cnt & (cnt - 1)) == 0) {
    const int sh = __ffs(cnt) - 1;
    for (int f = threadIdx.x; f < total; f += blockDim.x) {
      const int k = f >> sh, c = f & (cnt - 1);
      L.out[obase[c] + int64_t(k) * L.oks] = slots[c * PITCH + k];
    }
  } else {
    for (int f = threadIdx.x; f < total; f += blockDim.x) {
      const int k = f / cnt, c = f - k * cnt;
      L.out[obase[c] + int64_t(k) * L.oks] = slots[c * PITCH + k];
    }
  }
}

int fourstep_pass_e(int nl) { return nl <= 512 ? 16 : 32; }

bool fourstep_pass_supported(int nl) { return nl >= 64 && nl <= 4096 && (nl & (nl - 1)) == 0; }

int fourstep_pass_smem(int nl, int c) { return c * ((spad_len(nl) + 1) & ~1) * int(sizeof(float2)); }

template <int NL, int E, int DIR>
static cudaError_t run_fourstep(const FourStepLaunch& L, cudaStream_t st) {
  const int smem = fourstep_pass_smem(NL, L.c);
  {
    const cudaError_t e = ensure_dynamic_smem(reinterpret_cast<const void*>(fourstep_pass_kernel<NL, E, DIR>), smem);
    if (e != cudaSuccess) return e;
  }
  const int64_t blocks = (L.count + L.c - 1) / L.c;
  return launch_pdl(fourstep_pass_kernel<NL, E, DIR>, dim3(unsigned(blocks)), dim3((NL / E) * L.c), size_t(smem),
                    st, L);
}

cudaError_t launch_fourstep_pass(int nl, int dir, const FourStepLaunch& L, cudaStream_t st) {
#define PLFFT_B200_FS(NV, EV)                                                        \
  if (nl == NV) return dir < 0 ? run_fourstep<NV, EV, -1>(L, st) : run_fourstep<NV, EV, 1>(L, st);
  PLFFT_B200_FS(64, 16)
  PLFFT_B200_FS(128, 16)
  PLFFT_B200_FS(256, 16)
  PLFFT_B200_FS(512, 16)
  PLFFT_B200_FS(1024, 32)
  PLFFT_B200_FS(2048, 32)
  PLFFT_B200_FS(4096, 32)
#undef PLFFT_B200_FS
  return cudaErrorInvalidValue;
}

}  // namespace plfft_b200
