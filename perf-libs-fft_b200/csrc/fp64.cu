// FP64 data type (complex<double> / double), reference include/plfft.h:
// 143-154 with the FP32 conventions (docs/plfft.md:100-166).
//
// fp64_tile_kernel: one transform per CTA in shared memory, Stockham stages
// of radix 2..8 with FP64 twiddles from a host table (the same stage
// recurrence as the FP32 engine: butterfly j reads x[j + i n/R], multiplies
// by W_{Ns R}^{(j mod Ns) i}, writes y[(j / Ns) Ns R + j mod Ns + i Ns]);
// an optional four-step twiddle W_N^{col k} and a scale on the outputs.
// fp64_dft_kernel: direct O(n^2) sums with exactly reduced indices, for
// lengths without a smooth factorization.
// fp64_real_pre / fp64_real_post: R2C and C2R through a length-n complex
// transform (real input widened; Hermitian spectrum expanded).
#include "kernels.h"

namespace plfft_b200 {

__device__ __forceinline__ double2 dmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 dmulc(double2 a, double2 b) {  // a * conj(b)
  return make_double2(fma(a.x, b.x, a.y * b.y), fma(a.y, b.x, -a.x * b.y));
}

template <int DIR>
__global__ void __launch_bounds__(256) fp64_tile_kernel(const F64TileLaunch L) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int n = L.desc.n;
  double2* buf0 = reinterpret_cast<double2*>(smraw);
  double2* buf1 = buf0 + n;
  const int64_t g = blockIdx.x;
  const int64_t m = g / L.ia.ncols, col = g - (g / L.ia.ncols) * L.ia.ncols;
  const double2* x = L.in + m * L.ia.mdist + col * L.ia.cdist;
  for (int k = threadIdx.x; k < n; k += blockDim.x) buf0[k] = x[int64_t(k) * L.ia.kstride];
  __syncthreads();
  double2* src = buf0;
  double2* dst = buf1;
  for (int s = 0; s < L.desc.nstages; ++s) {
    const F64Stage st = L.desc.st[s];
    const int R = st.radix, ns = st.ns, nb = n / R;
    const double2* om = L.omega + st.om_off;  // exp(-2 pi i q / R), q < R
    for (int j = threadIdx.x; j < nb; j += blockDim.x) {
      double2 a[8];
      const int r = j % ns;
      for (int i = 0; i < R; ++i) {
        double2 v = src[j + i * nb];
        if (ns > 1 && i > 0) {
          const double2 w = L.tw[st.tw_off + (i - 1) * ns + r];
          v = DIR < 0 ? dmul(v, w) : dmulc(v, w);
        }
        a[i] = v;
      }
      const int base = (j / ns) * ns * R + r;
      for (int k = 0; k < R; ++k) {
        double2 acc = a[0];
        int idx = 0;
        for (int i = 1; i < R; ++i) {
          idx += k;
          if (idx >= R) idx -= R;
          acc.x += DIR < 0 ? a[i].x * om[idx].x - a[i].y * om[idx].y : a[i].x * om[idx].x + a[i].y * om[idx].y;
          acc.y += DIR < 0 ? a[i].x * om[idx].y + a[i].y * om[idx].x : a[i].y * om[idx].x - a[i].x * om[idx].y;
        }
        dst[base + k * ns] = acc;
      }
    }
    __syncthreads();
    double2* t = src;
    src = dst;
    dst = t;
  }
  const int64_t om_ = g / L.oa.ncols, ocol = g - om_ * L.oa.ncols;
  double2* y = L.out + om_ * L.oa.mdist + ocol * L.oa.cdist;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    double2 v = src[k];
    if (L.post.n != 0) {  // W_N^{col k} = lo[e mod L] * hi[e / L]
      const int64_t e = (col * k) % L.post.n;
      const double2 w = dmul(L.post.lo[e % L.post.l], L.post.hi[e / L.post.l]);
      v = DIR < 0 ? dmul(v, w) : dmulc(v, w);
    }
    y[int64_t(k) * L.oa.kstride] = make_double2(v.x * L.scale, v.y * L.scale);
  }
}

// direct sums: X_k = sum_j x_j W_n^{jk}, W from an n-entry table
template <int DIR>
__global__ void __launch_bounds__(256) fp64_dft_kernel(const F64TileLaunch L) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int n = L.desc.n;
  double2* xs = reinterpret_cast<double2*>(smraw);
  const int64_t g = blockIdx.x;
  const double2* x = L.in + g * L.ia.mdist;
  for (int k = threadIdx.x; k < n; k += blockDim.x) xs[k] = x[int64_t(k) * L.ia.kstride];
  __syncthreads();
  double2* y = L.out + g * L.oa.mdist;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    double2 acc = make_double2(0.0, 0.0);
    int idx = 0;
    for (int j = 0; j < n; ++j) {
      const double2 w = L.tw[idx];
      const double2 v = xs[j];
      acc.x += DIR < 0 ? v.x * w.x - v.y * w.y : v.x * w.x + v.y * w.y;
      acc.y += DIR < 0 ? v.x * w.y + v.y * w.x : v.y * w.x - v.x * w.y;
      idx += k;
      if (idx >= n) idx -= n;
    }
    y[int64_t(k) * L.oa.kstride] = make_double2(acc.x * L.scale, acc.y * L.scale);
  }
}

int fp64_tile_smem(int n) { return 2 * n * int(sizeof(double2)); }

cudaError_t launch_fp64_tile(int dir, bool direct, const F64TileLaunch& L, cudaStream_t st) {
  const int smem = direct ? L.desc.n * int(sizeof(double2)) : fp64_tile_smem(L.desc.n);
  auto kern = direct ? (dir < 0 ? fp64_dft_kernel<-1> : fp64_dft_kernel<1>)
                     : (dir < 0 ? fp64_tile_kernel<-1> : fp64_tile_kernel<1>);
  {
    const cudaError_t e = ensure_dynamic_smem(reinterpret_cast<const void*>(kern), smem);
    if (e != cudaSuccess) return e;
  }
  if (L.ntr <= 0) return cudaSuccess;
  kern<<<dim3(unsigned(L.ntr)), dim3(256), smem, st>>>(L);
  return cudaGetLastError();
}

// R2C: work[b][k] = (x_k, 0); C2R: work[b][k] = X_k for k <= n/2 and
// conj(X_{n-k}) above (imaginary parts of X_0 and X_{n/2} ignored)
__global__ void __launch_bounds__(256) fp64_real_pre(const F64RealLaunch L, int64_t m0, int64_t cnt) {
  const int64_t total = cnt * L.n;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t b = i / L.n, k = i - b * L.n, mb = m0 + b;
    double2 v;
    if (L.c2r == 0) {
      v = make_double2(static_cast<const double*>(L.in)[mb * L.idist + k * L.istride], 0.0);
    } else {
      const double2* X = static_cast<const double2*>(L.in) + mb * L.idist;
      const int64_t h = L.n / 2;
      if (k <= h) {
        v = X[k * L.istride];
        if (k == 0 || (k == h && L.n % 2 == 0)) v.y = 0.0;
      } else {
        const double2 c = X[(L.n - k) * L.istride];
        v = make_double2(c.x, -c.y);
      }
    }
    L.work[i] = v;
  }
}

// R2C: out[b][k] = work[b][k], k <= n/2; C2R: out[b][k] = Re work[b][k]
__global__ void __launch_bounds__(256) fp64_real_post(const F64RealLaunch L, int64_t m0, int64_t cnt) {
  const int64_t nout = L.c2r ? L.n : L.n / 2 + 1;
  const int64_t total = cnt * nout;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t b = i / nout, k = i - b * nout, mb = m0 + b;
    const double2 v = L.work[b * L.n + k];
    if (L.c2r)
      static_cast<double*>(L.out)[mb * L.odist + k * L.ostride] = v.x * L.scale;
    else
      static_cast<double2*>(L.out)[mb * L.odist + k * L.ostride] = make_double2(v.x * L.scale, v.y * L.scale);
  }
}

static unsigned fp64_grid(int64_t total) {
  const int64_t blocks = (total + 255) / 256;
  return unsigned(blocks < 148 * 16 ? (blocks > 0 ? blocks : 1) : 148 * 16);
}

cudaError_t launch_fp64_real(bool pre, const F64RealLaunch& L, int64_t m0, int64_t cnt, cudaStream_t st) {
  const int64_t nout = pre ? L.n : (L.c2r ? L.n : L.n / 2 + 1);
  if (pre)
    fp64_real_pre<<<fp64_grid(cnt * nout), 256, 0, st>>>(L, m0, cnt);
  else
    fp64_real_post<<<fp64_grid(cnt * nout), 256, 0, st>>>(L, m0, cnt);
  return cudaGetLastError();
}

}  // namespace plfft_b200
