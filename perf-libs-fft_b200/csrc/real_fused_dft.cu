// Fused real-data kernels: R2C/C2R and half-complex instantiations.
#include "real_fused.cuh"

namespace plfft_b200 {

cudaError_t launch_real_fused_dft(int kind, int m, const RealFusedLaunch& L, cudaStream_t st) {
  switch (kind) {
    case FR_R2C: return launch_real_fused_kind<FR_R2C>(m, L, st);
    case FR_C2R: return launch_real_fused_kind<FR_C2R>(m, L, st);
    case FR_R2HC: return launch_real_fused_kind<FR_R2HC>(m, L, st);
    case FR_HC2R: return launch_real_fused_kind<FR_HC2R>(m, L, st);
  }
  return cudaErrorNotSupported;
}

}  // namespace plfft_b200
