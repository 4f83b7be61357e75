// Power-of-two C2C FP32 kernels: host-side entry points.  The kernels and
// their launch logic are in c2c_pow2.cuh; each (elements per thread,
// direction) pair is instantiated in its own translation unit.
#include "kernels.h"
#include "stockham_desc.h"

namespace plfft_b200 {

cudaError_t launch_c2c_pow2_e16_fwd(int n, const Pow2Launch& L, cudaStream_t st);
cudaError_t launch_c2c_pow2_e16_inv(int n, const Pow2Launch& L, cudaStream_t st);
cudaError_t launch_c2c_pow2_e32_fwd(int n, const Pow2Launch& L, cudaStream_t st);
cudaError_t launch_c2c_pow2_e32_inv(int n, const Pow2Launch& L, cudaStream_t st);

int pow2_smem_bytes(int n, int g) { return g * ((spad_len(n) + 1) & ~1) * int(sizeof(float2)); }

bool pow2_supported(int n, int e) {
  if (e != 16 && e != 32) return false;
  if (n < 64 || n > 8192 || (n & (n - 1))) return false;
  return n / e <= (e <= 16 ? 512 : 256);
}

cudaError_t launch_c2c_pow2(int n, int e, int dir, const Pow2Launch& L, cudaStream_t st) {
  if (!pow2_supported(n, e)) return cudaErrorInvalidValue;
  if (e == 16) return dir < 0 ? launch_c2c_pow2_e16_fwd(n, L, st) : launch_c2c_pow2_e16_inv(n, L, st);
  return dir < 0 ? launch_c2c_pow2_e32_fwd(n, L, st) : launch_c2c_pow2_e32_inv(n, L, st);
}

}  // namespace plfft_b200
