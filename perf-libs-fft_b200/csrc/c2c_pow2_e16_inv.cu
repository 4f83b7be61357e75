// Power-of-two C2C kernels, 16 elements per thread, inverse direction.
#include "c2c_pow2.cuh"

namespace plfft_b200 {

cudaError_t launch_c2c_pow2_e16_inv(int n, const Pow2Launch& L, cudaStream_t st) {
  return launch_c2c_pow2_ed<16, 1>(n, L, st);
}

}  // namespace plfft_b200
