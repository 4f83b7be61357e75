// Launch descriptors shared by the host planner (plan.cpp) and the CUDA
// kernels.  Plain structs passed by value as kernel parameters.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "stockham_desc.h"

namespace plfft_b200 {

// Two-level twiddle for a four-step pass: W_N^e = lo[e % L] * hi[e / L].
struct TwoLevel {
  const float2* lo;
  const float2* hi;
  int64_t n;  // full transform length N (0: no four-step twiddle)
  int l;      // split point L
};

// Address of element k of transform g:
//   base + (g / ncols) * mdist + (g % ncols) * cdist + k * kstride
// (units: complex elements for complex data, scalars for real data).
struct Addr {
  int64_t mdist;
  int64_t cdist;
  int64_t kstride;
  int64_t ncols;
};

// Register-engine C2C launch: howmany transforms of length n, T = n/E
// threads each, G transforms per CTA.
struct RegLaunch {
  const float2* in;
  float2* out;
  int64_t howmany;
  int64_t istride, idist, ostride, odist;
  int t, g;
  float scale;
  FftDesc desc;
  const float2* tw;
};

// Shared-memory tile launch: C transforms per CTA, ntr transforms total,
// `nthr` threads per CTA.
struct TileLaunch {
  const float2* in;
  float2* out;
  int64_t ntr;
  Addr ia, oa;
  int c, nthr, ld;
  float scale;
  FftDesc desc;
  const float2* tw;
  TwoLevel post;  // four-step twiddle applied to outputs (k = output index,
                  // col = g % ia.ncols), if post.n != 0
};

// kernel entry points (c2c.cu)
cudaError_t launch_c2c_reg(int e, int dir, const RegLaunch& L, cudaStream_t st);
cudaError_t launch_c2c_tile(int maxe, int dir, const TileLaunch& L, cudaStream_t st);
int reg_smem_bytes(int n, int g);
int tile_smem_bytes(int ld, int c);

}  // namespace plfft_b200
