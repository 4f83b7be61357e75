// Stage list of one on-chip Stockham transform (host + device).
#pragma once

namespace plfft_b200 {

constexpr int kMaxStages = 20;

struct Stage {
  int radix;
  int ns;        // product of the earlier radices
  int ns_shift;  // log2(ns) if ns is a power of two, else -1
  int tw_off;    // offset of this stage's twiddle rows in the table
};

struct FftDesc {
  int n;
  int nstages;
  Stage st[kMaxStages];
};

// shared-memory row pitch for a transform of length n (odd, padded)
inline
#ifdef __CUDACC__
__host__ __device__
#endif
int spad_len(int n) { return (n + (n >> 4)) | 1; }

constexpr int spad_len_c(int n) { return (n + (n >> 4)) | 1; }

}  // namespace plfft_b200
