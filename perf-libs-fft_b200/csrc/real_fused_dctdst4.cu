// Fused real-data kernels: DCT-IV, DST-IV and DHT instantiations.
#include "real_fused.cuh"

namespace plfft_b200 {

cudaError_t launch_real_fused_dctdst4(int kind, int m, const RealFusedLaunch& L, cudaStream_t st) {
  switch (kind) {
    case FR_DCT4: return launch_real_fused_kind<FR_DCT4>(m, L, st);
    case FR_DST4: return launch_real_fused_kind<FR_DST4>(m, L, st);
    case FR_DHT: return launch_real_fused_kind<FR_DHT>(m, L, st);
  }
  return cudaErrorNotSupported;
}

}  // namespace plfft_b200
