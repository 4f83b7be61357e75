// Power-of-two C2C FP32 kernel with a compile-time stage list.
//
// N = R0 * E^(S-1): stage 0 is radix R0 (no twiddles), stages 1.. are radix E.
// T = N/E threads per transform, G transforms per CTA.  Unit-stride batches
// are moved by the TMA engine: one bulk copy per transform into shared memory
// (mbarrier completion, bounded wait), and one bulk copy back out after the
// result is written over the same shared-memory slots.  Between stages the
// data is exchanged through a padded shared-memory buffer; because every
// index is a compile-time power of two the address arithmetic folds to
// shifts and masks, and only the codelets this N uses are instantiated.
//
// This is the fast path for the reference's power-of-two C2C plans
// (src/planner/strategies/cooley_tukey.hpp:622-679 recursion of radix-r
// twiddle levels; here all levels of one transform stay on chip).
#pragma once
#include "kernels.h"
#include "launch_pdl.cuh"
#include "ptx.cuh"
#include "pow2_stages.cuh"

#include <algorithm>

namespace plfft_b200 {


template <int N, int E, int DIR>
__global__ void __launch_bounds__(pow2_max_threads<E>(), pow2_min_blocks<E>()) c2c_pow2_kernel(const Pow2Launch L) {
  using P = P2<N, E>;
  constexpr int T = P::T;
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ uint64_t bar;
  const int G = L.g;
  // one buffer per transform: bulk-copied input (natural order), then the
  // padded stage exchanges, then the natural-order result for the bulk store
  constexpr int PITCH = (spad_len_c(N) + 1) & ~1;  // even -> 16-byte aligned slots
  float2* inbuf = reinterpret_cast<float2*>(smraw);
  const int grp = threadIdx.x / T;
  const int t = threadIdx.x - grp * T;
  const int64_t b0 = int64_t(blockIdx.x) * G;
  const int64_t remain = L.howmany - b0;
  const int cnt = remain < G ? int(remain) : G;
  const bool live = grp < cnt;
  float2* mine = inbuf + grp * PITCH;
  float2* xb = mine;

  auto sync = [&]() {
    if constexpr (T <= 32)
      __syncwarp();
    else
      __syncthreads();
  };

  float2 v[E];
  if (L.tma_in) {
    if (threadIdx.x == 0) {
      mbar_init(&bar, 1);
      mbar_fence_init();
    }
    __syncthreads();
    const bool stall = int(blockIdx.x) == L.stall_cta;  // test hook: no loads
    if (threadIdx.x == 0 && !stall) {
      mbar_arrive_expect_tx(&bar, uint32_t(cnt) * N * 8u);
      for (int c = 0; c < cnt; ++c) bulk_g2s(inbuf + c * PITCH, L.in + (b0 + c) * L.idist, N * 8u, &bar);
    }
    const uint64_t lim = L.wait_ns ? L.wait_ns : kWaitLimitNs;
    const bool ok = mbar_wait_bounded(&bar, 0, lim);
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) {
        report_device_error(L.err, 1);
        // copies issued into this CTA's shared memory land before it exits
        if (!stall) mbar_wait_bounded(&bar, 0, lim);
      }
      return;
    }
    if (live) {
#pragma unroll
      for (int q = 0; q < E; ++q) v[q] = mine[t + T * q];
    } else {
#pragma unroll
      for (int q = 0; q < E; ++q) v[q] = make_float2(0.f, 0.f);
    }
  } else {
    if (live) {
      const float2* src = L.in + (b0 + grp) * L.idist;
#pragma unroll
      for (int q = 0; q < E; ++q) v[q] = src[t + T * q];
    } else {
#pragma unroll
      for (int q = 0; q < E; ++q) v[q] = make_float2(0.f, 0.f);
    }
  }

  st_bfly<T, E, P::radix(0), 1, 0, DIR>(v, t, L.tw);
  Stages<N, E, DIR, 1>::run(v, t, xb, L.tw, sync);

  const float s = L.scale;
  if (s != 1.f) {
#pragma unroll
    for (int q = 0; q < E; ++q) v[q] = cscale(v[q], s);
  }
  if (L.tma_out) {
    sync();  // last exchange fully read before the slots are reused
    if (live) {
#pragma unroll
      for (int q = 0; q < E; ++q) mine[t + T * q] = v[q];
    }
    fence_proxy_async();
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int c = 0; c < cnt; ++c) bulk_s2g(L.out + (b0 + c) * L.odist, inbuf + c * PITCH, N * 8u);
      bulk_commit();
      bulk_wait_read_all();
    }
  } else if (live) {
    float2* dst = L.out + (b0 + grp) * L.odist;
#pragma unroll
    for (int q = 0; q < E; ++q) dst[t + T * q] = v[q];
  }
}

// Persistent variant: each CTA owns a ring of R = L.slots buffer slots and
// walks the groups blockIdx.x, blockIdx.x + gridDim.x, ...  The bulk loads
// of the next R-1 groups are in flight while the current one is
// transformed, and each result leaves through an asynchronous bulk store.
// TWS: the stage twiddles are copied to shared memory once per CTA.
constexpr int kMaxSlots = 8;

template <int N, int E, int DIR, bool TWS>
__global__ void __launch_bounds__(pow2_max_threads<E>(), pow2_min_blocks<E>()) c2c_pow2_ring_kernel(const Pow2Launch L) {
  using P = P2<N, E>;
  constexpr int T = P::T;
  constexpr int PITCH = (spad_len_c(N) + 1) & ~1;
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ uint64_t bar[kMaxSlots];
  const int G = L.g;
  const int R = L.slots;
  const int64_t ngroups = (L.howmany + G - 1) / G;
  const int grp = threadIdx.x / T;
  const int t = threadIdx.x - grp * T;
  float2* const ring = reinterpret_cast<float2*>(smraw);
  float2* const tws = ring + R * G * PITCH;
  const float2* tw = TWS ? tws : L.tw;

  auto group_of = [&](int k) { return int64_t(blockIdx.x) + int64_t(k) * gridDim.x; };
  auto count_of = [&](int64_t g) {
    const int64_t r = L.howmany - g * G;
    return r < G ? int(r) : G;
  };
  auto slot = [&](int k) { return ring + (k % R) * G * PITCH; };
  const bool stall = int(blockIdx.x) == L.stall_cta;  // test hook: no loads
  const uint64_t lim = L.wait_ns ? L.wait_ns : kWaitLimitNs;
  uint32_t pending = 0;  // thread 0: slots with a load in flight
  auto issue = [&](int k) {  // thread 0 only
    const int64_t g = group_of(k);
    if (g >= ngroups || stall) return;
    const int cnt = count_of(g);
    pending |= 1u << (k % R);
    uint64_t* b = &bar[k % R];
    mbar_arrive_expect_tx(b, uint32_t(cnt) * N * 8u);
    float2* dst = slot(k);
    for (int c = 0; c < cnt; ++c) bulk_g2s(dst + c * PITCH, L.in + (g * G + c) * L.idist, N * 8u, b);
  };
  auto sync = [&]() {
    if constexpr (T <= 32)
      __syncwarp();
    else
      __syncthreads();
  };

  if (threadIdx.x == 0) {
    for (int b = 0; b < R; ++b) mbar_init(&bar[b], 1);
    mbar_fence_init();
  }
  __syncthreads();
  // launched programmatically (launch_pdl.cuh): the set-up above overlaps
  // the end of the previous launch; no global input is read and no output
  // written before that launch has completed
  griddep_wait();
  griddep_launch_dependents();
  // with direct stores a slot is free again right after its transform, so
  // all R slots hold loads in flight; with bulk stores one slot drains
  const int ahead = L.dstore ? R : R - 1;
  if (threadIdx.x == 0)
    for (int k = 0; k < ahead; ++k) issue(k);
  if constexpr (TWS) {
    for (int i = threadIdx.x; i < L.tw_len; i += blockDim.x) tws[i] = L.tw[i];
    __syncthreads();
  }
  for (int k = 0; group_of(k) < ngroups; ++k) {
    const int64_t g = group_of(k);
    const int cnt = count_of(g);
    const bool live = grp < cnt;
    float2* mine = slot(k) + grp * PITCH;
    const bool ok = mbar_wait_bounded(&bar[k % R], uint32_t(k / R) & 1u, lim);
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) {
        report_device_error(L.err, 1);
        // the load in flight in each slot belongs to the one group
        // j in [k, k + R) with j % R == slot: let them land before exiting
        for (int j = k; j < k + R; ++j)
          if (pending & (1u << (j % R))) mbar_wait_bounded(&bar[j % R], uint32_t(j / R) & 1u, lim);
      }
      break;
    }
    if (threadIdx.x == 0) pending &= ~(1u << (k % R));
    float2 v[E];
    if (live) {
#pragma unroll
      for (int q = 0; q < E; ++q) v[q] = mine[t + T * q];
    } else {
#pragma unroll
      for (int q = 0; q < E; ++q) v[q] = make_float2(0.f, 0.f);
    }
    st_bfly<T, E, P::radix(0), 1, 0, DIR, TWS>(v, t, tw);
    Stages<N, E, DIR, 1, TWS>::run(v, t, mine, tw, sync);
    const float s = L.scale;
    if (s != 1.f) {
#pragma unroll
      for (int q = 0; q < E; ++q) v[q] = cscale(v[q], s);
    }
    if (L.dstore) {
      // coalesced stores from registers; the slot is refilled at once
      if (live) {
        float2* dst = L.out + (g * G + grp) * L.odist;
#pragma unroll
        for (int q = 0; q < E; ++q) dst[t + T * q] = v[q];
      }
      __syncthreads();  // every read of this slot is done
      if (threadIdx.x == 0) {
        fence_proxy_async();
        issue(k + R);
      }
      continue;
    }
    sync();
    if (live) {
#pragma unroll
      for (int q = 0; q < E; ++q) mine[t + T * q] = v[q];
    }
    fence_proxy_async();
    __syncthreads();
    if (threadIdx.x == 0) {
      const float2* src = slot(k);
      for (int c = 0; c < cnt; ++c) bulk_s2g(L.out + (g * G + c) * L.odist, src + c * PITCH, N * 8u);
      bulk_commit();
      bulk_wait_read_but1();  // the slot of group k-1 is free again
      issue(k + R - 1);
    }
  }
  if (threadIdx.x == 0) bulk_wait_read_all();
}

// Warp-group variant: a persistent CTA holds GP independent groups of
// W = T/32 warps; each group transforms one sequence at a time through its
// own ring of NS shared-memory slots, with its own mbarriers and producer
// lane, so groups never wait on each other.  Group-local synchronisation is
// __syncwarp (W == 1) or a named barrier.  The stage twiddles are copied to
// shared memory once per CTA.  The refill of a slot is issued one iteration
// after its bulk store, so the store has drained before the slot is reused.
constexpr int kMaxGroups = 15;

template <int N, int E, int DIR, int NS>
__global__ void __launch_bounds__(512, 1) c2c_pow2_group_kernel(const Pow2Launch L) {
  using P = P2<N, E>;
  constexpr int T = P::T;
  static_assert(T % 32 == 0, "group kernel needs whole warps");
  constexpr int W = T / 32;
  constexpr int PITCH = (spad_len_c(N) + 1) & ~1;
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ uint64_t bar[kMaxGroups][NS];
  __shared__ int64_t meta[kMaxGroups][NS];  // transform held by each slot
  __shared__ int next;                      // CTA-local work counter
  const int grp = threadIdx.x / T;
  const int t = threadIdx.x - grp * T;
  float2* tws = reinterpret_cast<float2*>(smraw);
  float2* slots = tws + L.tw_len + ((L.tw_len & 1) ? 1 : 0);
  float2* myslots = slots + grp * NS * PITCH;
  // this CTA's contiguous share of the batch
  const int64_t lo = L.howmany * blockIdx.x / gridDim.x;
  const int64_t hi = L.howmany * (blockIdx.x + 1) / gridDim.x;
  const bool producer = (t == 0);
  const uint64_t lim = L.wait_ns ? L.wait_ns : kWaitLimitNs;
  uint32_t pending = 0;  // producer: slots with a load in flight

  auto gsync = [&]() {
    if constexpr (W == 1)
      __syncwarp();
    else
      asm volatile("bar.sync %0, %1;" ::"r"(grp + 1), "r"(T) : "memory");
  };
  // producer: claim the next transform of this CTA and start its load into
  // slot s (or mark the slot as the end of the group's work)
  auto fetch = [&](int s) {
    const int64_t b = lo + atomicAdd(&next, 1);
    meta[grp][s] = b;
    uint64_t* br = &bar[grp][s];
    if (b < hi) {
      pending |= 1u << s;
      mbar_arrive_expect_tx(br, N * 8u);
      bulk_g2s(myslots + s * PITCH, L.in + b * L.idist, N * 8u, br);
    } else {
      mbar_arrive(br);
    }
  };

  if (threadIdx.x == 0) next = 0;
  if (producer) {
    for (int s = 0; s < NS; ++s) mbar_init(&bar[grp][s], 1);
    mbar_fence_init();
  }
  __syncthreads();
  // start the rings first, then stage the twiddles while the loads fly
  if (producer)
    for (int s = 0; s < NS; ++s) fetch(s);
  for (int i = threadIdx.x; i < L.tw_len; i += blockDim.x) tws[i] = L.tw[i];
  __syncthreads();

  for (int k = 0;; ++k) {
    const int s = k % NS;
    const bool ok = mbar_wait_bounded(&bar[grp][s], uint32_t(k / NS) & 1u, lim);
    bool failed;
    if constexpr (W == 1) {
      failed = __any_sync(0xffffffffu, !ok);
    } else {
      uint32_t any;
      asm volatile(
          "{\n\t.reg .pred p, q;\n\t"
          "setp.ne.u32 p, %1, 0;\n\t"
          "bar.red.or.pred q, %2, %3, p;\n\t"
          "selp.u32 %0, 1, 0, q;\n\t}"
          : "=r"(any)
          : "r"(ok ? 0u : 1u), "r"(grp + 1), "r"(T)
          : "memory");
      failed = any != 0;
    }
    if (failed) {
      if (producer) {
        report_device_error(L.err, 1);
        // loads in flight belong to iterations j in [k, k + NS), one per slot
        for (int j = k; j < k + NS; ++j)
          if (pending & (1u << (j % NS))) mbar_wait_bounded(&bar[grp][j % NS], uint32_t(j / NS) & 1u, lim);
      }
      break;  // group-local exit; other groups are independent
    }
    if (producer) pending &= ~(1u << s);
    const int64_t b = meta[grp][s];
    if (b >= hi) break;
    float2* mine = myslots + s * PITCH;
    float2 v[E];
#pragma unroll
    for (int q = 0; q < E; ++q) v[q] = mine[t + T * q];
    st_bfly<T, E, P::radix(0), 1, 0, DIR, true>(v, t, tws);
    // the slot used by iteration k-1 has had a full stage to drain its store
    if (k >= 1 && producer) {
      bulk_wait_read_all();
      fetch((k - 1) % NS);
    }
    Stages<N, E, DIR, 1, true>::run(v, t, mine, tws, gsync);
    const float sc = L.scale;
    if (sc != 1.f) {
#pragma unroll
      for (int q = 0; q < E; ++q) v[q] = cscale(v[q], sc);
    }
    gsync();
#pragma unroll
    for (int q = 0; q < E; ++q) mine[t + T * q] = v[q];
    fence_proxy_async();
    gsync();
    if (producer) {
      bulk_s2g(L.out + b * L.odist, mine, N * 8u);
      bulk_commit();
    }
  }
  if (producer) bulk_wait_read_all();
}

inline int pow2_sm_count() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 1;
  }
  return n;
}

template <int N, int E, int DIR>
cudaError_t run_pow2(const Pow2Launch& L, cudaStream_t st) {
  const int threads = (N / E) * L.g;
  const int64_t ngroups = (L.howmany + L.g - 1) / L.g;
  if constexpr ((N / E) % 32 == 0) {
    if (L.tma_in && L.tma_out && L.ring >= 2) {
      constexpr int T = N / E;
      constexpr int PITCH = (spad_len_c(N) + 1) & ~1;
      const int ns = L.ring == 3 ? 3 : 2;
      const int per_group = ns * PITCH * 8;
      const int tw_bytes = ((L.tw_len + 1) & ~1) * 8;
      int gp = (227 * 1024 - 1024 - tw_bytes) / per_group;
      gp = std::min(gp, std::min(kMaxGroups, 512 / T));
      if (L.gp > 0) gp = std::min(gp, L.gp);  // explicit cap from the planner
      if (gp >= 1) {
        const int smem = tw_bytes + gp * per_group;
        const int64_t want_groups = L.howmany;
        const int64_t grid = std::max<int64_t>(1, std::min<int64_t>(pow2_sm_count(), (want_groups + gp - 1) / gp));
        auto launch = [&](auto kern) {
          cudaError_t e = ensure_dynamic_smem(reinterpret_cast<const void*>(kern), smem);
          if (e != cudaSuccess) return e;
          kern<<<dim3(unsigned(grid)), dim3(gp * T), smem, st>>>(L);
          return cudaGetLastError();
        };
        return ns == 3 ? launch(c2c_pow2_group_kernel<N, E, DIR, 3>) : launch(c2c_pow2_group_kernel<N, E, DIR, 2>);
      }
    }
  }
  if (L.tma_in && L.tma_out && L.ring) {
    if (L.slots < 2 || L.slots > kMaxSlots) return cudaErrorInvalidValue;
    auto* k = L.tws ? c2c_pow2_ring_kernel<N, E, DIR, true> : c2c_pow2_ring_kernel<N, E, DIR, false>;
    const int smem = L.slots * pow2_smem_bytes(N, L.g) + (L.tws ? ((L.tw_len + 1) & ~1) * 8 : 0);
    int per_sm = 0;
    cudaError_t e = cached_blocks_per_sm(reinterpret_cast<const void*>(k), threads, smem, &per_sm);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    // k groups per CTA so that the grid is one resident wave
    const int64_t cap = int64_t(per_sm) * pow2_sm_count();
    const int64_t per_cta = (ngroups + cap - 1) / cap;
    const int64_t grid = (ngroups + per_cta - 1) / per_cta;
    return launch_pdl(k, dim3(unsigned(grid)), dim3(threads), size_t(smem), st, L);
  }
  const int smem = pow2_smem_bytes(N, L.g);
  {
    cudaError_t e = ensure_dynamic_smem(reinterpret_cast<const void*>(c2c_pow2_kernel<N, E, DIR>), smem);
    if (e != cudaSuccess) return e;
  }
  c2c_pow2_kernel<N, E, DIR><<<dim3(unsigned(ngroups)), dim3(threads), smem, st>>>(L);
  return cudaGetLastError();
}

// the lengths 64..8192 at E elements per thread in direction DIR
// (instantiated in c2c_pow2_e{16,32}_{fwd,inv}.cu, compiled in parallel)
template <int E, int DIR>
cudaError_t launch_c2c_pow2_ed(int n, const Pow2Launch& L, cudaStream_t st) {
  switch (n) {
    case 64: return run_pow2<64, E, DIR>(L, st);
    case 128: return run_pow2<128, E, DIR>(L, st);
    case 256: return run_pow2<256, E, DIR>(L, st);
    case 512: return run_pow2<512, E, DIR>(L, st);
    case 1024: return run_pow2<1024, E, DIR>(L, st);
    case 2048: return run_pow2<2048, E, DIR>(L, st);
    case 4096: return run_pow2<4096, E, DIR>(L, st);
    case 8192: return run_pow2<8192, E, DIR>(L, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace plfft_b200
