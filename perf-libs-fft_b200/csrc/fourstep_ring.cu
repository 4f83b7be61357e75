// Power-of-two four-step passes on dense batches, moved by the TMA engine.
//
// The same two passes as fourstep.cu (the reference's twiddled Cooley-Tukey
// levels, src/level_ac_t_c2c.cpp:50-85 and src/level_ab_t_c2c.cpp:49-80),
// for batches whose members have unit stride:
//   pass 0 (columns): a tile is C adjacent columns of one member, all NL = n1
//     rows: tensor-map boxes of C x 256 elements (C*8-byte rows) in, the
//     column FFTs and W_n^{column * k1}, the same boxes out;
//   pass 1 (rows): a tile is C adjacent rows of NL = n2 elements (one bulk
//     copy of C*NL*8 contiguous bytes); the results leave transposed,
//     X[k1 + n1 k2], as tensor-map boxes of C consecutive k1 by 256 k2.
// With C*8 = 128, 64 or 32 bytes the boxes use the matching shared-memory
// swizzle, so the C groups reading one column each hit distinct banks.  CTAs
// are persistent and walk their tiles through a ring of R slots: the loads of
// the next R-2 tiles and the stores of the previous one are in flight while a
// tile is transformed.  Thread 0 issues the copies; every wait on a copy is
// bounded.  No copy uses cluster multicast.
//
// Slot layout: the row form (element (k, c) at byte k*C*8 + c*8, swizzled)
// holds pass-0 inputs and both passes' outputs; pass-1 inputs are dense rows
// (group c at c*NL), and the stage exchanges use the group form (group c at
// c*PITCH, padded as in pow2_stages.cuh).  A tile is moved into registers
// before its slot is reused for the exchanges.
#include <algorithm>

#include "kernels.h"
#include "launch_pdl.cuh"
#include "pow2_stages.cuh"
#include "ptx.cuh"

namespace plfft_b200 {

constexpr int kFsRingMaxSlots = 4;
constexpr int kFsBoxRows = 256;  // tensor-map box limit per dimension

template <int NL, int C>
struct FsRingShape {
  static constexpr int PITCH = (spad_len_c(NL) + 1) & ~1;
  static constexpr int ROWS = NL * C;  // row form, complex elements
  static constexpr int GROUPS = C * PITCH;
  static constexpr int BYTES = (ROWS > GROUPS ? ROWS : GROUPS) * 8;
  static constexpr int SLOT = (BYTES + 1023) & ~1023;  // bytes; slots stay 1024-aligned for the swizzle
  // the swizzle of a C*8-byte row: 16-byte chunk bits [4, 4+b) ^= bits [7, 7+b)
  static constexpr int SWZ = C == 16 ? 7 : C == 8 ? 3 : 1;
};

template <int C>
__device__ __forceinline__ int fs_swz(int byte_off) {
  constexpr int MASK = C == 16 ? 7 : C == 8 ? 3 : 1;
  return byte_off ^ (((byte_off >> 7) & MASK) << 4);
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, int x, int y, int z, const void* src) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(x), "r"(y), "r"(z), "r"(smem_addr(src))
               : "memory");
}

template <int NL, int E, int DIR, int PASS, int C>
__global__ void __launch_bounds__(C*(NL / E)) fourstep_ring_kernel(const __grid_constant__ FourStepRingLaunch L) {
  using P = P2<NL, E>;
  using S = FsRingShape<NL, C>;
  constexpr int T = P::T;
  constexpr int NB = NL > kFsBoxRows ? NL / kFsBoxRows : 1;  // boxes per tile
  constexpr int BR = NL / NB;                                // rows per box
  extern __shared__ __align__(1024) unsigned char smraw[];
  __shared__ uint64_t bar[kFsRingMaxSlots];
  const int R = L.slots;
  const int grp = threadIdx.x / T;
  const int t = threadIdx.x - grp * T;
  // the dynamic window starts 1024-aligned (the launch adds 1 KB of slack)
  unsigned char* const base =
      smraw + ((1024u - (smem_addr(smraw) & 1023u)) & 1023u);
  auto slot = [&](int k) { return base + (k % R) * S::SLOT; };
  auto tile_of = [&](int k) { return int64_t(blockIdx.x) + int64_t(k) * gridDim.x; };
  const uint64_t lim = L.wait_ns ? L.wait_ns : kWaitLimitNs;
  uint32_t pending = 0;  // thread 0: slots with a load in flight
  auto sync = [&]() {
    if constexpr (T <= 32)
      __syncwarp();
    else
      __syncthreads();
  };
  // thread 0: start the loads of tile k into its slot
  auto issue = [&](int k) {
    const int64_t g = tile_of(k);
    if (g >= L.tiles) return;
    const int m = int(g / L.blocks);
    const int blk = int(g - int64_t(m) * L.blocks);
    uint64_t* b = &bar[k % R];
    unsigned char* dst = slot(k);
    pending |= 1u << (k % R);
    mbar_arrive_expect_tx(b, uint32_t(C) * NL * 8u);
    if constexpr (PASS == 0) {
#pragma unroll
      for (int r = 0; r < NB; ++r) tma_load_3d(dst + r * BR * C * 8, &L.tm_in, blk * C, r * BR, m, b);
    } else {
      bulk_g2s(dst, L.in + int64_t(m) * L.idist + int64_t(blk) * C * NL, uint32_t(C) * NL * 8u, b);
    }
  };

  if (threadIdx.x == 0) {
    for (int i = 0; i < R; ++i) mbar_init(&bar[i], 1);
    mbar_fence_init();
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&L.tm_out)) : "memory");
    if constexpr (PASS == 0) asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&L.tm_in)) : "memory");
  }
  __syncthreads();
  griddep_wait();  // launched programmatically (launch_pdl.cuh)
  griddep_launch_dependents();
  if (threadIdx.x == 0)
    for (int k = 0; k < R - 1; ++k) issue(k);
  const int lshift = __ffs(L.post.l) - 1;

  for (int k = 0; tile_of(k) < L.tiles; ++k) {
    const int64_t g = tile_of(k);
    const int m = int(g / L.blocks);
    const int blk = int(g - int64_t(m) * L.blocks);
    const bool ok = mbar_wait_bounded(&bar[k % R], uint32_t(k / R) & 1u, lim);
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) {
        report_device_error(L.err, 1);
        // the load in flight in each slot belongs to the one tile j in
        // [k, k + R) with j % R == slot: let them land before exiting
        for (int j = k; j < k + R; ++j)
          if (pending & (1u << (j % R))) mbar_wait_bounded(&bar[j % R], uint32_t(j / R) & 1u, lim);
      }
      break;
    }
    if (threadIdx.x == 0) pending &= ~(1u << (k % R));
    unsigned char* const s = slot(k);
    float2* const mine = reinterpret_cast<float2*>(s) + grp * S::PITCH;
    float2 v[E];
    if constexpr (PASS == 0) {
#pragma unroll
      for (int q = 0; q < E; ++q)
        v[q] = *reinterpret_cast<const float2*>(s + fs_swz<C>(((t + T * q) * C + grp) * 8));
    } else {
      const float2* row = reinterpret_cast<const float2*>(s) + grp * NL;
#pragma unroll
      for (int q = 0; q < E; ++q) v[q] = row[t + T * q];
    }
    st_bfly<T, E, P::radix(0), 1, 0, DIR>(v, t, L.tw);
    __syncthreads();  // every group has its inputs before the exchange regions (which overlap them) are written
    Stages<NL, E, DIR, 1>::run(v, t, mine, L.tw, sync);
    if constexpr (PASS == 0) {
      // W_n^{col k1}, k1 = t + T q: a table lookup every fourth q and a
      // product with W_n^{col T} in between
      const uint32_t col = uint32_t(blk * C + grp);
      const uint32_t e1 = col * uint32_t(T);
      const float2 step =
          cmul(__ldg(L.post.lo + (e1 & uint32_t(L.post.l - 1))), __ldg(L.post.hi + (e1 >> lshift)));
      float2 w = make_float2(1.f, 0.f);
#pragma unroll
      for (int q = 0; q < E; ++q) {
        if ((q & 3) == 0) {
          const uint32_t e = col * uint32_t(t + T * q);
          w = cmul(__ldg(L.post.lo + (e & uint32_t(L.post.l - 1))), __ldg(L.post.hi + (e >> lshift)));
        } else {
          w = cmul(w, step);
        }
        v[q] = twmul<DIR>(v[q], w);
      }
    }
    if (L.scale != 1.f) {
#pragma unroll
      for (int q = 0; q < E; ++q) v[q] = cscale(v[q], L.scale);
    }
    __syncthreads();  // every group's exchanges are done before the row form is written
#pragma unroll
    for (int q = 0; q < E; ++q) *reinterpret_cast<float2*>(s + fs_swz<C>(((t + T * q) * C + grp) * 8)) = v[q];
    fence_proxy_async();
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
      for (int r = 0; r < NB; ++r) tma_store_3d(&L.tm_out, blk * C, r * BR, m, s + r * BR * C * 8);
      bulk_commit();
      bulk_wait_read_but1();  // the stores of tile k-1 have left its slot
      issue(k + R - 1);
    }
  }
  if (threadIdx.x == 0) bulk_wait_read_all();
}

// sub-transform lengths 128..1024 (the halves of n = 2^14..2^20); tile widths:
// 16 or 8 columns (128- or 64-byte rows) up to nl = 512, 8 or 4 at 1024
bool fourstep_ring_supported(int nl, int c) {
  if (nl < 128 || nl > 1024 || (nl & (nl - 1))) return false;
  return nl <= 512 ? (c == 16 || c == 8) : (c == 8 || c == 4);
}

int fourstep_ring_smem(int nl, int c, int slots) {
  const int pitch = (spad_len(nl) + 1) & ~1;
  const int bytes = std::max(nl * c, c * pitch) * 8;
  return slots * ((bytes + 1023) & ~1023) + 1024;
}

static int fs_ring_sm_count() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 1;
  }
  return n;
}

template <int NL, int E, int DIR, int PASS, int C>
static cudaError_t run_fourstep_ring(const FourStepRingLaunch& L, cudaStream_t st) {
  auto* k = fourstep_ring_kernel<NL, E, DIR, PASS, C>;
  if (L.slots < 2 || L.slots > kFsRingMaxSlots) return cudaErrorInvalidValue;
  const int threads = C * (NL / E);
  const int smem = L.slots * FsRingShape<NL, C>::SLOT + 1024;
  int per_sm = 0;
  cudaError_t e = cached_blocks_per_sm(reinterpret_cast<const void*>(k), threads, smem, &per_sm);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  const int64_t cap = int64_t(per_sm) * fs_ring_sm_count();
  const int64_t grid = std::min<int64_t>(L.tiles, cap);
  return launch_pdl(k, dim3(unsigned(grid)), dim3(threads), size_t(smem), st, L);
}

template <int NL, int E, int C>
static cudaError_t run_fourstep_ring_dp(int dir, int pass, const FourStepRingLaunch& L, cudaStream_t st) {
  if (pass == 0)
    return dir < 0 ? run_fourstep_ring<NL, E, -1, 0, C>(L, st) : run_fourstep_ring<NL, E, 1, 0, C>(L, st);
  return dir < 0 ? run_fourstep_ring<NL, E, -1, 1, C>(L, st) : run_fourstep_ring<NL, E, 1, 1, C>(L, st);
}

cudaError_t launch_fourstep_ring(int nl, int c, int dir, int pass, const FourStepRingLaunch& L, cudaStream_t st) {
  if (L.tiles <= 0) return cudaSuccess;
  if (!fourstep_ring_supported(nl, c)) return cudaErrorInvalidValue;
#define PLFFT_B200_FSR(NV, EV, CV) \
  if (nl == NV && c == CV) return run_fourstep_ring_dp<NV, EV, CV>(dir, pass, L, st);
  PLFFT_B200_FSR(128, 16, 16)
  PLFFT_B200_FSR(256, 16, 16)
  PLFFT_B200_FSR(512, 16, 16)
  PLFFT_B200_FSR(128, 16, 8)
  PLFFT_B200_FSR(256, 16, 8)
  PLFFT_B200_FSR(512, 16, 8)
  PLFFT_B200_FSR(1024, 32, 8)
  PLFFT_B200_FSR(1024, 32, 4)
#undef PLFFT_B200_FSR
  return cudaErrorInvalidValue;
}

}  // namespace plfft_b200
