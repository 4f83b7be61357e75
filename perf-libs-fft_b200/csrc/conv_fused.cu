// One-kernel Rader and Bluestein transforms: the whole convolution of one
// member stays on chip.
//
// Both algorithms reduce a length-n DFT to a cyclic convolution (reference
// src/planner/strategies/bluestein.hpp:37-240 and
// src/planner/strategies/rader.hpp:36-254).  Here the convolution is done
// with power-of-two FFTs of length M held in registers (the Stockham stage
// list of pow2_stages.cuh), so one launch does, per member,
//   load (+ chirp or generator permutation) -> FFT_M -> x spectrum ->
//   IFFT_M -> (chirp or inverse permutation) + scale -> store,
// reading the n inputs once and writing the n outputs once.
//
// Bluestein, with w_k = exp(dir i pi (k^2 mod 2n) / n) and M >= 2n - 1:
//   a_j = x_j w_j (j < n, 0 up to M),  c = IFFT_M(FFT_M(a) * B),  y_k = c_k w_k,
//   B = FFT_M(b)/M,  b_m = conj(w_|m|) for |m| < n, placed cyclically.
// Rader, for prime P, generator g, L = P - 1 and M >= 2L - 1: the length-L
// cyclic convolution is computed as a zero-padded length-M one,
//   a_q = x[g^q mod P] (q < L, 0 up to M),  A = FFT_M(a),  A0 = A[0],
//   c = IFFT_M(A * B),  y[g^-m mod P] = x_0 + c_m (m < L),  y_0 = x_0 + A0,
//   B = FFT_M(b')/M,  b'_j = b_j (j < L), b'_{M-j} = b_{L-j} (0 < j < L),
//   b_q = exp(dir 2 pi i g^-q / P).
// Inputs and outputs pass through the member's shared-memory buffer so the
// global loads and stores stay coalesced (Rader permutes there).
#include <utility>
#include <vector>

#include "kernels.h"
#include "stockham_desc.h"

namespace plfft_b200 {

cudaError_t launch_conv_fused_rader(int m, int e, int minb, const ConvFusedLaunch& L, cudaStream_t st);
cudaError_t launch_conv_fused_bluestein(int m, int e, int minb, const ConvFusedLaunch& L, cudaStream_t st);

std::vector<std::pair<int, int>> conv_fused_shapes(int m) {
  switch (m) {
    case 64:
    case 128:
    case 256:
    case 512: return {{16, 3}};
    case 1024: return {{32, 2}, {16, 3}};
    case 2048: return {{16, 3}, {32, 2}};
    case 4096: return {{16, 4}, {16, 3}, {32, 2}};
    case 8192: return {{32, 2}};
    default: return {};
  }
}

int conv_fused_smem_bytes(int m, int g) { return g * ((spad_len_c(m) + 1) & ~1) * int(sizeof(float2)); }

bool conv_fused_supported(int m, int e, int minb) {
  for (const auto& sh : conv_fused_shapes(m))
    if (sh.first == e && sh.second == minb) return true;
  return false;
}

cudaError_t launch_conv_fused(int m, int e, int minb, bool rader, const ConvFusedLaunch& L, cudaStream_t st) {
  if (L.howmany <= 0) return cudaSuccess;
  if (!conv_fused_supported(m, e, minb)) return cudaErrorInvalidValue;
  return rader ? launch_conv_fused_rader(m, e, minb, L, st) : launch_conv_fused_bluestein(m, e, minb, L, st);
}

}  // namespace plfft_b200
