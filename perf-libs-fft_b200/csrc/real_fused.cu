// Fused single-kernel real transforms for N = 2M, M a power of two: host-side
// entry points.  The kernel and its launch logic are in real_fused.cuh; the
// kinds are instantiated in three translation units compiled in parallel.
#include "kernels.h"

namespace plfft_b200 {

cudaError_t launch_real_fused_dft(int kind, int m, const RealFusedLaunch& L, cudaStream_t st);
cudaError_t launch_real_fused_dctdst23(int kind, int m, const RealFusedLaunch& L, cudaStream_t st);
cudaError_t launch_real_fused_dctdst4(int kind, int m, const RealFusedLaunch& L, cudaStream_t st);

int real_fused_e(int m) {
  if (m <= 512) return 16;
  if (m <= 2048) return 32;
  if (m == 4096) return 16;
  return 32;
}

bool real_fused_supported(int m) { return m >= 64 && m <= 8192 && (m & (m - 1)) == 0; }

cudaError_t launch_real_fused(int kind, int m, const RealFusedLaunch& L, cudaStream_t st) {
  if (!real_fused_supported(m)) return cudaErrorInvalidValue;
  for (auto f : {launch_real_fused_dft, launch_real_fused_dctdst23, launch_real_fused_dctdst4}) {
    const cudaError_t e = f(kind, m, L, st);
    if (e != cudaErrorNotSupported) return e;
  }
  return cudaErrorInvalidValue;
}

}  // namespace plfft_b200
