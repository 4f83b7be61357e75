// Fused real-data kernels: DCT-II/III and DST-II/III instantiations.
#include "real_fused.cuh"

namespace plfft_b200 {

cudaError_t launch_real_fused_dctdst23(int kind, int m, const RealFusedLaunch& L, cudaStream_t st) {
  switch (kind) {
    case FR_DCT2: return launch_real_fused_kind<FR_DCT2>(m, L, st);
    case FR_DST2: return launch_real_fused_kind<FR_DST2>(m, L, st);
    case FR_DCT3: return launch_real_fused_kind<FR_DCT3>(m, L, st);
    case FR_DST3: return launch_real_fused_kind<FR_DST3>(m, L, st);
  }
  return cudaErrorNotSupported;
}

}  // namespace plfft_b200
