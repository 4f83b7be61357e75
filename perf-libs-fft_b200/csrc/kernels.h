// Launch descriptors shared by the host planner (plan.cpp) and the CUDA
// kernels.  Plain structs passed by value as kernel parameters.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <utility>
#include <vector>

#include "stockham_desc.h"

namespace plfft_b200 {

// Two-level twiddle for a four-step pass: W_N^e = lo[e % L] * hi[e / L].
struct TwoLevel {
  const float2* lo;
  const float2* hi;
  int64_t n;  // full transform length N (0: no four-step twiddle)
  int l;      // split point L
};

// Address of element k of transform g:
//   base + (g / ncols) * mdist + (g % ncols) * cdist + k * kstride
// (units: complex elements for complex data, scalars for real data).
struct Addr {
  int64_t mdist;
  int64_t cdist;
  int64_t kstride;
  int64_t ncols;
};

// Register-engine C2C launch: howmany transforms of length n, T = n/E
// threads each, G transforms per CTA.
struct RegLaunch {
  const float2* in;
  float2* out;
  int64_t howmany;
  int64_t istride, idist, ostride, odist;
  int t, g;
  float scale;
  FftDesc desc;
  const float2* tw;
};

// Shared-memory tile launch: C transforms per CTA, ntr transforms total,
// `nthr` threads per CTA.
struct TileLaunch {
  const float2* in;
  float2* out;
  int64_t ntr;
  Addr ia, oa;
  int c, nthr, ld;
  float scale;
  FftDesc desc;
  const float2* tw;
  TwoLevel post;  // four-step twiddle applied to outputs (k = output index,
                  // col = g % ia.ncols), if post.n != 0
};

// Static power-of-two C2C launch (c2c_pow2.cu): unit element stride,
// transforms idist/odist apart, G per CTA; bulk copies when aligned.
struct Pow2Launch {
  const float2* in;
  float2* out;
  int64_t howmany;
  int64_t idist, odist;
  int g;
  float scale;
  const float2* tw;
  int tw_len;  // entries in tw
  int tma_in, tma_out;
  int ring;  // 0 one-shot CTAs, 1 CTA ring, 2/3 warp-group rings (slots)
  int slots;  // CTA ring: buffer slots (2..8), loads run slots-1 groups ahead
  int tws;    // CTA ring: stage twiddles copied to shared memory
  int dstore; // CTA ring: results stored from registers (no bulk store)
  int gp;    // warp-group kernel: groups per CTA (0 = as many as fit)  // persistent ring-buffered variant
  int* err;  // host-mapped status word: set to 1 if a bounded device wait ran out
  uint64_t wait_ns;  // limit of each bounded wait (0: kWaitLimitNs)
  int stall_cta;     // test hook: this CTA issues no loads, so its first wait runs out (-1: none)
};

// Real-data transforms through a complex DFT of length `len`
// (realwrap.cu): pre-kernel builds the complex sequence in `work`, a C2C plan
// transforms it in place, the post-kernel extracts the outputs.
enum RealWrapKind {
  RW_R2C = 0,
  RW_C2R = 1,
  RW_DCT1 = 2,
  RW_DCT2 = 3,
  RW_DCT3 = 4,
  RW_DCT4 = 5,
  RW_DST1 = 6,
  RW_DST2 = 7,
  RW_DST3 = 8,
  RW_DST4 = 9,
  RW_DHT = 10,
  RW_R2HC = 11,
  RW_HC2R = 12
};
// Elementwise weights that turn a transform into the adjoint of another
// (input weights applied by the pre-kernel, output weights by the post-kernel)
enum AdjointWeight {
  AW_NONE = 0,
  AW_HERM_HALF = 1,    // complex bins 0 < k < n/2 times 1/2
  AW_HERM_DOUBLE = 2,  // complex bins 0 < k < n/2 times 2
  AW_FIRST_X2 = 3,     // element 0 times 2
  AW_FIRST_HALF = 4,   // element 0 times 1/2
  AW_LAST_X2 = 5,      // element n-1 times 2
  AW_LAST_HALF = 6,    // element n-1 times 1/2
  AW_INNER_HALF = 7,   // elements 0 < j < n-1 times 1/2
  AW_INNER_X2 = 8,     // elements 0 < j < n-1 times 2
  AW_HC_HALF = 9,      // half-complex entries other than 0 and n/2 times 1/2
  AW_HC_DOUBLE = 10    // half-complex entries other than 0 and n/2 times 2
};
struct RealWrapLaunch {
  const void* in;
  void* out;
  void* work;  // [chunk][len] complex (float2, or double2 when fp64)
  int64_t n, len, nout;
  int64_t istride, idist, ostride, odist;
  double scale;
  int wmode_in, wmode_out;
  int fp64;  // 0: FP32 data, 1: FP64 data
};
cudaError_t launch_realwrap(bool pre, int kind, const RealWrapLaunch& L, int64_t m0, int64_t cnt,
                            cudaStream_t st);
// Half-length R2C / C2R (realwrap.cu) for even n = 2m, FP32: the split after
// (R2C) or the merge before (C2R) a length-m C2C over the member's real data
// read as complex pairs.  Distances and strides in complex elements of the
// complex side; work holds m complex per member of the chunk.
struct RealHalfLaunch {
  const float2* in;  // C2R: the complex input
  float2* out;       // R2C: the complex output
  float2* work;      // [chunk][m]
  int64_t m;
  int64_t istride, idist, ostride, odist;
  float scale;
  int wmode_in, wmode_out;  // AdjointWeight modes over the n-point spectrum
  const float2* tw;         // W_n^k, k = 0..m
};
cudaError_t launch_real_half(bool r2c, const RealHalfLaunch& L, int64_t m0, int64_t cnt, cudaStream_t st);

// Rader / Bluestein elementwise passes (conv.cu).  n: transform length,
// m: convolution length (M for Bluestein, P-1 for Rader).
enum ConvStep {
  CONV_BS_PRE = 0,
  CONV_MUL = 1,
  CONV_MUL_SAVE0 = 2,
  CONV_BS_POST = 3,
  CONV_RD_PRE = 4,
  CONV_RD_POST = 5
};
struct ConvLaunch {
  const float2* in;
  float2* out;
  float2* work;   // [chunk][m]
  float2* sum0;   // [chunk] (Rader: A[0] per member)
  const float2* chirp;  // Bluestein w_k, k < n
  const float2* spec;   // convolution spectrum, m entries
  const int* perm_in;   // Rader g^q mod P
  const int* perm_out;  // Rader g^-q mod P
  int64_t n, m;
  int64_t istride, idist, ostride, odist;
  float scale;
};
cudaError_t launch_conv(int step, const ConvLaunch& L, int64_t m0, int64_t cnt, cudaStream_t st);

// One-kernel Rader / Bluestein over power-of-two convolution lengths
// 64 <= m <= 8192 (conv_fused.cu)
struct ConvFusedLaunch {
  const float2* in;
  float2* out;
  int64_t howmany, istride, idist, ostride, odist;
  int n;                // transform length (the prime P for Rader)
  int g;                // members per CTA
  const float2* tw;     // stage twiddles of the length-m power-of-two stage list
  const float2* chirp;  // Bluestein w_k, k < n
  const float2* spec;   // FFT_m(b) / m
  const int* perm_in;   // Rader g^q mod P, q < P - 1
  const int* perm_out;  // Rader g^-q mod P
  float scale;
};
// Shape of a launch: e elements per thread (16 or 32) and minb, the resident
// 256-thread CTAs per SM the register allocation is sized for (2, 3, 4:
// 128, 85, 64 registers per thread).  conv_fused_shapes(m) lists the
// instantiated shapes for m, the default first.
std::vector<std::pair<int, int>> conv_fused_shapes(int m);
bool conv_fused_supported(int m, int e, int minb);
int conv_fused_smem_bytes(int m, int g);
cudaError_t launch_conv_fused(int m, int e, int minb, bool rader, const ConvFusedLaunch& L, cudaStream_t st);

// Grouped mixed-length execution (grouped.cu)
enum GTaskType { GT_TILE = 0, GT_RADER = 1, GT_BLUE = 2 };
enum GOp {
  GO_NONE = 0,
  GO_GATHER = 1,      // prologue: x[perm_in[e]]
  GO_CHIRP = 2,       // prologue: x[e] * tab[e] (0 for e >= len); epilogue: y * tab[e], e < len only
  GO_TWIDDLE = 3,     // epilogue: four-step twiddle W^{col * k}
  GO_SPEC = 4,        // epilogue: y * tab[e]
  GO_SPEC_SAVE0 = 5,  // epilogue: save y at e == 0, then y * tab[e]
  GO_SCATTER = 6      // epilogue: out[perm_out[e]] = x0 + y, out[0] = x0 + saved
};
constexpr int kGroupBuffers = 3;  // 0 user input, 1 user output, 2 workspace
struct GTask {
  int type, dir, n, cnt, desc;
  int in_buf, out_buf, aux_buf;
  int pre_op, post_op;
  int pre_len, post_len;
  int64_t in_off, out_off, aux_off;
  int64_t icdist, ikstride, ocdist, okstride;
  int64_t ie0, iec, iek, oe0, oec, oek;
  int64_t col0;
  const float2* pre_tab;
  const float2* post_tab;
  const float2* post_tab2;
  const int* perm_in;
  const int* perm_out;
  float2* sum0;
  TwoLevel tw2;
  float scale;
};
struct GroupPhase {
  const GTask* tasks;
  int ntasks;
  const FftDesc* descs;
  const float2* const* tws;
  float2* bases[kGroupBuffers];
  int* counter;
  int* done;
};
cudaError_t launch_grouped(const GroupPhase& P, int grid, int smem_bytes, cudaStream_t st);
int grouped_blocks_per_sm(int smem_bytes);
int group_max_smem_elems();

// Fused single-kernel real transforms for N = 2M, M a power of two
// (real_fused.cu).  Distances count elements of each buffer's own type.
enum FusedRealKind { FR_R2C = 0, FR_C2R = 1, FR_DCT2 = 2, FR_DST2 = 3, FR_DCT3 = 4, FR_DST3 = 5, FR_DCT4 = 6, FR_DST4 = 7,
                     FR_R2HC = 8, FR_HC2R = 9, FR_DHT = 10 };
struct RealFusedLaunch {
  const void* in;
  void* out;
  int64_t howmany, idist, odist;
  int g;  // transforms per CTA
  float scale;
  const float2* tw;    // stage twiddles of the length-M complex FFT
  const float2* post;  // W_N^k, k = 0..M (DCT-IV / DST-IV: exp(i pi p / N), p < M)
  const float2* rot;   // exp(-i pi k / 2N), k = 0..M (DCT-IV / DST-IV: exp(i pi (4q+1) / 4N), q < M)
  int pairs_in, pairs_out;  // real data may be moved as aligned float pairs
  int quads_in;             // real input may be read as aligned float4
  int e;                    // elements per thread of the length-M FFT
  int wmode;                // adjoint weights: 1 C2R input bins 0<k<M times 1/2,
                            // 2 R2C output bins 0<k<M times 2, 3 DCT-III input
                            // element 0 (DST-III: element N-1) times 2
};
bool real_fused_supported(int m);
int real_fused_e(int m);
cudaError_t launch_real_fused(int kind, int m, const RealFusedLaunch& L, cudaStream_t st);

// One pass of a power-of-two four-step transform (fourstep.cu): `count`
// sub-transforms of length nl, sub-transform g = (member g / ncols, column
// g % ncols), element k at base + member*mdist + column*cd + k*ks.
struct FourStepLaunch {
  const float2* in;
  float2* out;
  int64_t count, ncols;
  int64_t imdist, icd, iks;
  int64_t omdist, ocd, oks;
  int c;  // sub-transforms per CTA
  float scale;
  const float2* tw;  // stage twiddles of length nl
  TwoLevel post;     // W_n^{column * k} on the outputs when post.n != 0
};
bool fourstep_pass_supported(int nl);

// Dense-batch four-step passes moved by the TMA engine (fourstep_ring.cu):
// persistent CTAs over `tiles` = members * blocks tiles of c sub-transforms,
// a ring of `slots` shared-memory slots.  Pass 0: tile (m, b) is columns
// [b c, b c + c) of member m, loaded and stored through the tensor maps
// tm_in / tm_out (dims {n2, n1, members}), W_n^{col k} applied (post);
// pass 1: tile (m, b) is rows [b c, b c + c) of member m (nl contiguous
// elements each, from `in` with member distance idist), stored transposed
// through tm_out (dims {n1, n2, members}).
struct alignas(64) FourStepRingLaunch {
  CUtensorMap tm_in;   // pass 0 input
  CUtensorMap tm_out;  // output of either pass
  const float2* in;    // pass 1 input
  int64_t tiles, blocks;
  int64_t idist;
  int slots;
  float scale;
  const float2* tw;  // stage twiddles of length nl
  TwoLevel post;     // pass 0 only (pass 1: l = 1)
  int* err;          // host-mapped status word: set to 1 if a bounded device wait ran out
  uint64_t wait_ns;  // limit of each bounded wait (0: kWaitLimitNs)
};
bool fourstep_ring_supported(int nl, int c);
int fourstep_ring_smem(int nl, int c, int slots);
cudaError_t launch_fourstep_ring(int nl, int c, int dir, int pass, const FourStepRingLaunch& L, cudaStream_t st);
// 3-D tensor map over 8-byte elements: dims {d0, d1, d2}, byte strides of
// dims 1 and 2, box {b0, b1, 1}, shared-memory swizzle for b0*8-byte rows
cudaError_t encode_tensor_map_c64(CUtensorMap* map, const void* base, uint64_t d0, uint64_t d1, uint64_t d2,
                                  uint64_t stride1_bytes, uint64_t stride2_bytes, uint32_t b0, uint32_t b1);
int fourstep_pass_e(int nl);
int fourstep_pass_smem(int nl, int c);
cudaError_t launch_fourstep_pass(int nl, int dir, const FourStepLaunch& L, cudaStream_t st);

// Fixed-point C2C (fixed_point.cu), Q0.15 (bits 16) and Q0.7 (bits 8):
// power-of-two n <= 4096; one complex element is one storage word (int32
// for two int16, int16 for two int8); strides in elements.
struct FixedLaunch {
  const void* in;
  void* out;
  int64_t howmany;
  int64_t istride, idist, ostride, odist;
  const short4* tw;   // n >= 32: outer radix-16 level, per row j >= 1 and input i >= 1: (c, s, cvt(-s), c)
  const short4* tw2;  // n >= 512: inner radix-16 level over n / 256 rows, same layout
};
bool fixed_supported(int64_t n);
cudaError_t launch_fixed(int bits, int n, int dir, const FixedLaunch& L, cudaStream_t st);
// fixed-point R2C (forward), power-of-two n in [2, 4096]: input reals (int16
// or int8 lanes; istride / idist in reals), output bins 0..n/2 (packed
// complex; ostride / odist in complex elements); tw / tw2 as for the C2C
cudaError_t launch_fixed_r2c(int bits, int n, const FixedLaunch& L, cudaStream_t st);
// fixed-point C2R (backward), power-of-two n in [2, 4096]: input bins 0..n/2
// (packed complex; istride / idist in complex elements), output reals
// (ostride / odist in reals); tw / tw2: the backward tables
cudaError_t launch_fixed_c2r(int bits, int n, const FixedLaunch& L, cudaStream_t st);

// Split-BF16 tensor-core pass (split_bf16.cu): same addressing as a
// four-step pass, on-chip length nl in {256, 4096} as radix-16 DFT-matrix
// products; dftm = three 32x32 bf16 splits of the real DFT-16 matrix.
bool split_bf16_pass_supported(int nl);
int split_bf16_pass_c(int nl);
cudaError_t launch_split_bf16_pass(int nl, int dir, const FourStepLaunch& L, const uint32_t* dftm,
                                   cudaStream_t st);

// Single-pass four-step for n = 256 x 256 on an 8-CTA cluster
// (fourstep_cluster.cu); any strides, members idist/odist apart.
struct FourStepClusterLaunch {
  const float2* in;
  float2* out;
  int64_t howmany;
  int64_t istride, idist, ostride, odist;
  float scale;
  const float2* tw;  // stage twiddles of the 256-point FFT
  TwoLevel tw2;      // W_n^{c k1}
};
int fourstep_cluster_smem();
int fourstep_cluster_capacity();
cudaError_t launch_fourstep_cluster(int dir, const FourStepClusterLaunch& L, int max_clusters, cudaStream_t st);

// FP16 data type (half_io.cu): strided binary16 <-> dense FP32 chunk;
// comps = 1 (real) or 2 (complex) scalars per element.
cudaError_t launch_half_gather(const void* src, float* dense, int64_t m0, int64_t cnt, int64_t n, int64_t stride,
                               int64_t dist, int comps, cudaStream_t st);
cudaError_t launch_half_scatter(const float* dense, void* dst, int64_t m0, int64_t cnt, int64_t n, int64_t stride,
                                int64_t dist, int comps, cudaStream_t st);

// FP64 data type (fp64.cu)
struct F64Stage {
  int radix, ns, tw_off, om_off;
};
struct F64Desc {
  int n, nstages;
  F64Stage st[24];
};
struct TwoLevel64 {
  const double2* lo;
  const double2* hi;
  int64_t n;  // 0: no four-step twiddle
  int64_t l;
};
struct F64TileLaunch {
  const double2* in;
  double2* out;
  int64_t ntr;     // transforms (one per CTA)
  Addr ia, oa;     // element addressing, as the FP32 tile launch
  double scale;
  F64Desc desc;    // n and stages (direct kernel: n only)
  const double2* tw;     // stage twiddles (direct kernel: W_n^m, m < n)
  const double2* omega;  // exp(-2 pi i q / R) for each stage radix
  TwoLevel64 post;       // W_N^{col k} on the outputs when post.n != 0
};
struct F64RealLaunch {
  const void* in;
  void* out;
  double2* work;  // [cnt][n] complex
  int64_t n, istride, idist, ostride, odist;
  int c2r;
  double scale;
};
int fp64_tile_smem(int n);
cudaError_t launch_fp64_tile(int dir, bool direct, const F64TileLaunch& L, cudaStream_t st);
cudaError_t launch_fp64_real(bool pre, const F64RealLaunch& L, int64_t m0, int64_t cnt, cudaStream_t st);

// launch-time query caches (launch_cache.cpp)
cudaError_t ensure_dynamic_smem(const void* kernel, int bytes);
cudaError_t cached_blocks_per_sm(const void* kernel, int threads, int smem, int* blocks);

// kernel entry points (c2c.cu)
cudaError_t launch_c2c_reg(int e, int dir, const RegLaunch& L, cudaStream_t st);
cudaError_t launch_c2c_tile(int maxe, int dir, const TileLaunch& L, cudaStream_t st);
int reg_smem_bytes(int n, int g);
int tile_smem_bytes(int ld, int c);

// c2c_pow2.cu
bool pow2_supported(int n, int e);
int pow2_smem_bytes(int n, int g);
cudaError_t launch_c2c_pow2(int n, int e, int dir, const Pow2Launch& L, cudaStream_t st);

}  // namespace plfft_b200
