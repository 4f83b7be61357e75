// Programmatic dependent launch for the hot kernels.
//
// A kernel launched this way may have its CTAs placed on SMs while the
// previous kernel in the stream drains, so launch latency and the kernel's
// own set-up overlap that kernel's last CTAs.  Every kernel launched through
// launch_pdl calls griddep_wait() (ptx.cuh) before its first global read or
// write, which holds it until the previous kernel has completed and its
// writes are visible: stream order is unchanged for the data.
// PLFFT_B200_NO_PDL=1 launches without the attribute.
#pragma once

#include <cuda_runtime.h>

#include <cstdlib>
#include <utility>

namespace plfft_b200 {

inline bool pdl_enabled() {
  static const bool on = std::getenv("PLFFT_B200_NO_PDL") == nullptr;
  return on;
}

template <class... Params, class... Args>
cudaError_t launch_pdl(void (*kern)(Params...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                       Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl_enabled() ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

}  // namespace plfft_b200
