// Bluestein instantiations of the fused convolution kernel.
#include "conv_fused.cuh"

namespace plfft_b200 {

cudaError_t launch_conv_fused_bluestein(int m, int e, int minb, const ConvFusedLaunch& L, cudaStream_t st) {
  return launch_conv_fused_alg<false>(m, e, minb, L, st);
}

}  // namespace plfft_b200
