// plfft_cuda_c2c_execute_noalloc: a four-step C2C FP32 transform that makes
// no device allocation of any kind.
//
// Who needs it: callers that must not allocate device memory while they run,
// e.g. an application whose framework has already reserved the GPU's memory
// through its own pool (a cudaMalloc from this library would fail or fragment
// that pool), or a latency-critical loop in which cudaMalloc/cudaFree would
// synchronize the device.  Plan-based execution allocates its tables and its
// workspace with cudaMalloc when the plan is created; this entry point needs
// neither a plan nor a workspace.
//
// Where its memory comes from: the intermediate buffer of the four-step
// algorithm and the twiddle tables live in one file-scope device array,
// g_noalloc_scratch (kNoAllocBytes, 17 MiB).  Every GPU that loads the
// library holds this array until the process exits.  Host code cannot use
// the array's name as a device address (in host code it names a host-side
// stand-in), so the first call on each device, with that device current,
// looks the address up with cudaGetSymbolAddress and caches it.  That
// set-up happens inside the first call; make the first call on a device
// before any stream capture begins.
//
// Sharing: all calls on a device use the same array, and each call rewrites
// the parts it reads (tables first, then the intermediate buffer), so nothing
// carries over from the previous call.  Calls whose execution overlaps on the
// GPU (different streams without ordering between them) race on the array
// and must not be issued.
//
// Cost per call: one table-fill launch, then two launches per chunk of
// members (a chunk is as many members as fit the 16 MiB buffer), all on the
// caller's stream.  After the first call on a device the cached address is
// read without taking a lock.  The cache lives as long as the process's
// context on that device: after cudaDeviceReset the next call must not be
// made through this entry point until the process restarts, since the array
// is re-created at a new address.
#include <cuda_runtime.h>

#include <atomic>
#include <mutex>

#include "../../include/plfft.h"
#include "../../include/plfft_cuda.h"
#include "kernels.h"
#include "plan.hpp"
#include "stockham.cuh"

namespace plfft_b200 {

// intermediate buffer: the four-step scratch for a chunk of members
constexpr size_t kNoAllocWorkBytes = size_t(16) << 20;
// twiddle tables: stage rows of both passes and the two-level root tables
constexpr size_t kNoAllocTableBytes = size_t(1) << 20;
constexpr size_t kNoAllocBytes = kNoAllocWorkBytes + kNoAllocTableBytes;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kNoAllocMaxDevices = 64;
static std::mutex g_noalloc_mu;
static std::atomic<void*> g_noalloc_addr[kNoAllocMaxDevices] = {};

// device address of g_noalloc_scratch on the current device (looked up once
// per device, under a lock; later calls read it without one)
static cudaError_t noalloc_scratch(int dev, unsigned char** out) {
  if (dev < 0 || dev >= kNoAllocMaxDevices) return cudaErrorInvalidDevice;
  void* p = g_noalloc_addr[dev].load(std::memory_order_acquire);
  if (!p) {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    p = g_noalloc_addr[dev].load(std::memory_order_relaxed);
    if (!p) {
      const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess) return e;
      g_noalloc_addr[dev].store(p, std::memory_order_release);
    }
  }
  *out = static_cast<unsigned char*>(p);
  return cudaSuccess;
}

// stage list of an on-chip transform without building its twiddle values
static FftDesc noalloc_desc(int n, const std::vector<int>& radices, int* tw_count) {
  FftDesc d{};
  d.n = n;
  d.nstages = int(radices.size());
  int ns = 1, off = 0;
  for (size_t s = 0; s < radices.size(); ++s) {
    Stage& st = d.st[s];
    st.radix = radices[s];
    st.ns = ns;
    st.ns_shift = (ns & (ns - 1)) == 0 ? __builtin_ctz(unsigned(ns)) : -1;
    st.tw_off = off;
    if (ns > 1) off += (radices[s] - 1) * ns;
    ns *= radices[s];
  }
  *tw_count = off;
  return d;
}

// exp(-2 pi i k / m), evaluated in FP64 (table generation only)
__device__ __forceinline__ float2 noalloc_root(int64_t k, int64_t m) {
  k %= m;
  double s, c;
  sincospi(2.0 * double(k) / double(m), &s, &c);
  return make_float2(float(c), float(-s));
}

__device__ __forceinline__ void noalloc_stage_entry(float2* tw, const FftDesc& d, int f) {
  for (int s = 0; s < d.nstages; ++s) {
    const Stage& st = d.st[s];
    if (st.ns <= 1) continue;
    const int cnt = (st.radix - 1) * st.ns;
    if (f >= st.tw_off && f < st.tw_off + cnt) {
      const int g = f - st.tw_off;
      const int i = g / st.ns + 1;
      const int r = g - (i - 1) * st.ns;
      tw[f] = noalloc_root(int64_t(r) * i, int64_t(st.ns) * st.radix);
      return;
    }
  }
}

__global__ void __launch_bounds__(256) noalloc_fill_tables(float2* tw1, FftDesc d1, int n_tw1, float2* tw2, FftDesc d2,
                                                           int n_tw2, float2* lo, float2* hi, int64_t n, int l,
                                                           int n_hi) {
  const int total = n_tw1 + n_tw2 + l + n_hi;
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < total; f += gridDim.x * blockDim.x) {
    if (f < n_tw1) {
      noalloc_stage_entry(tw1, d1, f);
    } else if (f < n_tw1 + n_tw2) {
      noalloc_stage_entry(tw2, d2, f - n_tw1);
    } else if (f < n_tw1 + n_tw2 + l) {
      const int i = f - n_tw1 - n_tw2;
      lo[i] = noalloc_root(i, n);
    } else {
      const int i = f - n_tw1 - n_tw2 - l;
      hi[i] = noalloc_root(int64_t(i) * l, n);
    }
  }
}

static size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

}  // namespace plfft_b200

using namespace plfft_b200;

extern "C" plfft_status_t plfft_cuda_c2c_execute_noalloc(const void* d_input, void* d_output, int64_t n,
                                                        int64_t howmany, plfft_direction_t direction, void* stream) {
  if (!d_input || !d_output) return PLFFT_NULL_ARGUMENT;
  if (direction != PLFFT_FORWARD && direction != PLFFT_BACKWARD) return PLFFT_INVALID_TRANSFORM_KIND;
  if (howmany < 1) return PLFFT_UNSUPPORTED_BATCH;
  // the four-step range: longer than one on-chip pass, one member must fit
  // the static intermediate buffer
  if (n <= kMaxOnChip || n > int64_t(kNoAllocWorkBytes / sizeof(float2)) || !is_smooth(n)) return PLFFT_INVALID_SIZE;
  const int64_t n1 = four_step_split(n);
  if (!n1) return PLFFT_INVALID_SIZE;
  const int64_t n2 = n / n1;

  TileChoice t1, t2;
  if (!choose_tile(n1, true, t1) || !choose_tile(n2, false, t2)) return PLFFT_INVALID_SIZE;
  int ntw1 = 0, ntw2 = 0;
  const FftDesc d1 = noalloc_desc(int(n1), t1.radices, &ntw1);
  const FftDesc d2 = noalloc_desc(int(n2), t2.radices, &ntw2);
  int lbits = 0;
  while ((int64_t(1) << lbits) < n) ++lbits;
  const int l = 1 << ((lbits + 1) / 2);
  const int n_hi = int((n + l - 1) / l);
  const size_t table_bytes = align256(size_t(ntw1) * 8) + align256(size_t(ntw2) * 8) + align256(size_t(l) * 8) +
                             align256(size_t(n_hi) * 8);
  if (table_bytes > kNoAllocTableBytes) return PLFFT_INVALID_SIZE;

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return PLFFT_CUDA_ERROR;
  unsigned char* base = nullptr;
  if (noalloc_scratch(dev, &base) != cudaSuccess) return PLFFT_CUDA_ERROR;
  float2* work = reinterpret_cast<float2*>(base);
  unsigned char* tab = base + kNoAllocWorkBytes;
  float2* tw1 = reinterpret_cast<float2*>(tab);
  float2* tw2 = reinterpret_cast<float2*>(tab + align256(size_t(ntw1) * 8));
  float2* lo = reinterpret_cast<float2*>(tab + align256(size_t(ntw1) * 8) + align256(size_t(ntw2) * 8));
  float2* hi = reinterpret_cast<float2*>(reinterpret_cast<unsigned char*>(lo) + align256(size_t(l) * 8));
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  const int fill_total = ntw1 + ntw2 + l + n_hi;
  noalloc_fill_tables<<<(fill_total + 255) / 256, 256, 0, st>>>(tw1, d1, ntw1, tw2, d2, ntw2, lo, hi, n, l, n_hi);
  if (cudaGetLastError() != cudaSuccess) return PLFFT_CUDA_ERROR;

  // pass 1: columns (length n1, stride n2) times W_n^{n2 k1} into the
  // intermediate buffer; pass 2: rows (length n2), stored transposed
  TileLaunch a{};
  a.desc = d1;
  a.tw = tw1;
  a.ia = Addr{n, 1, n2, n2};
  a.oa = Addr{n, 1, n2, n2};
  a.c = t1.c;
  a.nthr = t1.nthr;
  a.ld = t1.ld;
  a.scale = 1.0f;
  a.post = TwoLevel{lo, hi, n, l};
  TileLaunch b{};
  b.desc = d2;
  b.tw = tw2;
  b.ia = Addr{n, n2, 1, n1};
  b.oa = Addr{n, 1, n1, n1};
  b.c = t2.c;
  b.nthr = t2.nthr;
  b.ld = t2.ld;
  b.scale = 1.0f;
  b.post = TwoLevel{nullptr, nullptr, 0, 1};

  const int64_t chunk = std::max<int64_t>(1, int64_t(kNoAllocWorkBytes / sizeof(float2)) / n);
  const float2* x = static_cast<const float2*>(d_input);
  float2* y = static_cast<float2*>(d_output);
  for (int64_t m0 = 0; m0 < howmany; m0 += chunk) {
    const int64_t cnt = std::min(chunk, howmany - m0);
    TileLaunch p = a;
    p.in = x + m0 * n;
    p.out = work;
    p.ntr = cnt * n2;
    if (launch_c2c_tile(t1.maxe, int(direction), p, st) != cudaSuccess) return PLFFT_CUDA_ERROR;
    TileLaunch q = b;
    q.in = work;
    q.out = y + m0 * n;
    q.ntr = cnt * n1;
    if (launch_c2c_tile(t2.maxe, int(direction), q, st) != cudaSuccess) return PLFFT_CUDA_ERROR;
  }
  return PLFFT_OK;
}
