// Planner: radix factorization, device twiddle tables and C2C schedules.
#include "plan.hpp"

#include <algorithm>
#include <atomic>
#include <cstring>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <sstream>

namespace plfft_b200 {

// ---------------------------------------------------------------------------
// number theory helpers
// ---------------------------------------------------------------------------
bool is_prime(int64_t n) {
  if (n < 2) return false;
  for (int64_t d = 2; d * d <= n; ++d)
    if (n % d == 0) return false;
  return true;
}

bool is_smooth(int64_t n) {
  if (n < 1) return false;
  for (int p : {2, 3, 5, 7, 11, 13})
    while (n % p == 0) n /= p;
  return n == 1;
}

// Split n into radices <= max_radix, largest first.  Mirrors the intent of
// the reference's factorize_descending (src/factorize.hpp:95-111): greedy
// division by the largest available kernel size.  The radix menu here is the
// set of on-chip codelets {16, 8, 4, 2, 13, 11, 7, 5, 3} (32 in the register
// engine).
std::vector<int> factor_radices(int64_t n, int max_radix) {
  std::vector<int> r;
  const int pow2_menu[] = {32, 16, 8, 4, 2};
  for (int p : pow2_menu) {
    if (p > max_radix) continue;
    while (n % p == 0) {
      r.push_back(p);
      n /= p;
    }
  }
  for (int p : {13, 11, 7, 5, 3}) {
    while (n % p == 0) {
      r.push_back(p);
      n /= p;
    }
  }
  if (n != 1) r.clear();
  return r;
}

void unit_root(int64_t k, int64_t n, double& c, double& s) {
  // cos/sin of 2 pi k / n with octant reduction in integers so that the
  // argument handed to libm is small and exact symmetry points are exact
  k %= n;
  if (k < 0) k += n;
  const long double kpi = 3.141592653589793238462643383279502884L;
  __int128 k8 = (__int128)8 * k;
  int64_t oct = int64_t(k8 / n);
  int64_t rem = int64_t(k8 - (__int128)oct * n);
  long double r = (long double)rem / (long double)n * (kpi / 4.0L);
  long double c0, s0;
  if (oct % 2 == 0) {
    c0 = cosl(r);
    s0 = sinl(r);
  } else {
    long double r2 = kpi / 4.0L - r;
    c0 = cosl(r2);
    s0 = -sinl(r2);
    oct += 1;
  }
  int64_t q = (oct / 2) % 4;
  long double cc = c0, ss = s0;
  if (q == 1) { cc = -s0; ss = c0; }
  if (q == 2) { cc = -c0; ss = -s0; }
  if (q == 3) { cc = s0; ss = -c0; }
  c = double(cc);
  s = double(ss);
}

static float2 root_f(int64_t k, int64_t n, int sign) {
  double c, s;
  unit_root(k, n, c, s);
  return make_float2(float(c), float(sign * s));
}

FftDesc make_desc(int n, const std::vector<int>& radices, std::vector<float2>& tw) {
  FftDesc d{};
  d.n = n;
  d.nstages = int(radices.size());
  int ns = 1;
  for (size_t s = 0; s < radices.size(); ++s) {
    const int R = radices[s];
    Stage& st = d.st[s];
    st.radix = R;
    st.ns = ns;
    st.ns_shift = (ns & (ns - 1)) == 0 ? __builtin_ctz(unsigned(ns)) : -1;
    st.tw_off = int(tw.size());
    if (ns > 1) {
      // rows i = 1..R-1, entry r: exp(-2 pi i r i / (ns R))
      for (int i = 1; i < R; ++i)
        for (int r = 0; r < ns; ++r) tw.push_back(root_f(int64_t(r) * i, int64_t(ns) * R, -1));
    }
    ns *= R;
  }
  return d;
}

static int ilog2(int64_t n) {
  int l = 0;
  while ((int64_t(1) << l) < n) ++l;
  return l;
}
static bool is_pow2(int64_t n) { return n > 0 && (n & (n - 1)) == 0; }

// ---------------------------------------------------------------------------
// register-engine C2C node
// ---------------------------------------------------------------------------
struct RegChoice {
  int e = 0, t = 0, g = 0;
  std::vector<int> radices;
};

static int env_int(const char* name, int dflt) {
  const char* v = std::getenv(name);
  return v ? std::atoi(v) : dflt;
}

static bool choose_reg(int64_t n, RegChoice& rc) {
  if (!is_pow2(n) || n < 64 || n > kMaxOnChip) return false;
  rc.e = env_int("PLFFT_B200_REG_E", n >= 1024 ? 32 : 16);
  if (n / rc.e > 256) return false;  // CTA limit of the register kernel
  int64_t rest = n;
  std::vector<int> big;
  while (rest % rc.e == 0 && rest >= rc.e) {
    big.push_back(rc.e);
    rest /= rc.e;
  }
  rc.radices.clear();
  if (rest > 1) rc.radices.push_back(int(rest));
  rc.radices.insert(rc.radices.end(), big.begin(), big.end());
  rc.t = int(n / rc.e);
  rc.g = env_int("PLFFT_B200_REG_G", std::max(1, 256 / rc.t));
  if (rc.g * rc.t > 256) rc.g = std::max(1, 256 / rc.t);
  while (rc.g > 1 && reg_smem_bytes(int(n), rc.g) > 100 * 1024) rc.g /= 2;
  return true;
}

struct C2CRegNode : Node {
  RegLaunch base{};
  int e = 0, dir = -1;
  DevBuf tw;
  std::vector<int> radices;
  cudaError_t run(const void* in, void* out, void*, cudaStream_t st) const override {
    RegLaunch L = base;
    L.in = static_cast<const float2*>(in);
    L.out = static_cast<float2*>(out);
    return launch_c2c_reg(e, dir, L, st);
  }
  std::string describe() const override {
    std::ostringstream o;
    o << "(c2c-reg n=" << base.desc.n << " e=" << e << " t=" << base.t << " g=" << base.g
      << " radices=";
    for (size_t i = 0; i < radices.size(); ++i) o << (i ? "x" : "") << radices[i];
    o << ")";
    return o.str();
  }
};

// ---------------------------------------------------------------------------
// static power-of-two C2C node (bulk-copy staged, compile-time radices)
// ---------------------------------------------------------------------------
// explicit launch shape (0 / -1: planner default or environment override)
struct Pow2Params {
  int e = 0, ring = -1, g = 0, gp = -1, slots = 0, tws = -1, dstore = -1;
};

struct C2CPow2Node : Node {
  Pow2Launch base{};
  int n = 0, e = 0, dir = -1;
  DevBuf tw;
  HostWord status;
  // test hook (PLFFT_B200_TEST_STALL_CTA): the CTA whose first load is
  // withheld in the next run only
  mutable std::atomic<int> stall_once{-1};
  uint64_t stall_wait_ns = 0;  // the shortened wait limit of that run
  void status_words(std::vector<int*>& out) const override { out.push_back(status.p); }
  cudaError_t run(const void* in, void* out, void*, cudaStream_t st) const override {
    Pow2Launch L = base;
    L.stall_cta = stall_once.exchange(-1);
    if (L.stall_cta >= 0) L.wait_ns = stall_wait_ns;
    L.in = static_cast<const float2*>(in);
    L.out = static_cast<float2*>(out);
    const bool dist_in_ok = L.howmany == 1 || (L.idist % 2) == 0;
    const bool dist_out_ok = L.howmany == 1 || (L.odist % 2) == 0;
    L.tma_in = (reinterpret_cast<uintptr_t>(in) % 16 == 0) && dist_in_ok;
    L.tma_out = (reinterpret_cast<uintptr_t>(out) % 16 == 0) && dist_out_ok;
    return launch_c2c_pow2(n, e, dir, L, st);
  }
  std::string describe() const override {
    std::ostringstream o;
    o << "(c2c-pow2 n=" << n << " e=" << e << " g=" << base.g;
    if (base.ring == 1)
      o << " ring slots=" << base.slots << (base.tws ? " tw-smem" : "") << (base.dstore ? " direct-store" : "");
    if (base.ring >= 2) o << " group-ring" << base.ring << " gp=" << base.gp;
    o << " bulk-copy)";
    return o.str();
  }
};

static int pow2_default_e(int64_t n) {
  if (n <= 512) return 16;
  if (n <= 2048) return 32;
  if (n == 4096) return 16;
  return 32;
}

static std::unique_ptr<Node> make_pow2(int64_t n, const Layout& lay, int dir, float scale, std::string* why,
                                       const Pow2Params& pp = Pow2Params{}) {
  int e = pp.e ? pp.e : env_int("PLFFT_B200_POW2_E", pow2_default_e(n));
  if (!pow2_supported(int(n), e)) e = pow2_default_e(n);
  if (!pow2_supported(int(n), e)) return nullptr;
  auto node = std::make_unique<C2CPow2Node>();
  node->n = int(n);
  node->e = e;
  node->dir = dir;
  // radices: leftover factor first, then radix-e stages
  std::vector<int> radices;
  int64_t rest = n;
  int ke = 0;
  while (rest % e == 0 && rest > 1) {
    rest /= e;
    ++ke;
  }
  if (rest > 1) radices.push_back(int(rest));
  for (int i = 0; i < ke; ++i) radices.push_back(e);
  std::vector<float2> tw;
  make_desc(int(n), radices, tw);
  if (node->tw.upload(tw) != cudaSuccess || node->status.alloc() != cudaSuccess) {
    if (why) *why = "device allocation failed";
    return nullptr;
  }
  const int t = int(n / e);
  int g = std::max(1, pp.g ? pp.g : env_int("PLFFT_B200_POW2_G", std::max(1, 32 / t)));
  const int maxthr = e <= 16 ? 512 : 256;
  while (g > 1 && (g * t > maxthr || pow2_smem_bytes(int(n), g) > 200 * 1024)) g /= 2;
  node->base.howmany = lay.howmany;
  node->base.idist = lay.idist;
  node->base.odist = lay.odist;
  node->base.g = g;
  node->base.scale = scale;
  node->base.tw = node->tw.as<float2>();
  node->base.tw_len = int(tw.size());
  node->base.err = node->status.device();
  node->base.wait_ns = 0;
  node->base.stall_cta = -1;
  // Test hook for the device-timeout path: PLFFT_B200_TEST_STALL_CTA=k makes
  // CTA k of this plan's first run withhold its loads, so its bounded wait
  // (PLFFT_B200_TEST_WAIT_US microseconds) runs out and the run reports
  // PLFFT_DEVICE_TIMEOUT; nothing is in flight when that CTA leaves.
  if (const char* v = std::getenv("PLFFT_B200_TEST_STALL_CTA")) {
    node->stall_once = std::atoi(v);
    node->stall_wait_ns = uint64_t(std::max(1, env_int("PLFFT_B200_TEST_WAIT_US", 2000))) * 1000u;
  }
  // CTA ring, one transform per CTA for n = 1024 (g = 32 / T), 3 slots:
  // measured best at batch 4096 (4.09 TB/s; deeper rings, twiddles in
  // shared memory, register stores and the warp-group rings were slower)
  node->base.ring = pp.ring >= 0 ? pp.ring : env_int("PLFFT_B200_POW2_RING", 1);
  node->base.gp = std::max(0, pp.gp >= 0 ? pp.gp : env_int("PLFFT_B200_POW2_GP", 0));
  node->base.slots = std::min(8, std::max(2, pp.slots ? pp.slots : env_int("PLFFT_B200_POW2_SLOTS", 3)));
  node->base.tws = pp.tws >= 0 ? pp.tws : env_int("PLFFT_B200_POW2_TWS", 0);
  node->base.dstore = pp.dstore >= 0 ? pp.dstore : env_int("PLFFT_B200_POW2_DS", 0);
  // the ring's slots must fit in shared memory
  while (node->base.slots > 2 &&
         node->base.slots * pow2_smem_bytes(int(n), g) + node->base.tws * int(tw.size() + 1) * 8 > 200 * 1024)
    --node->base.slots;
  return node;
}

// ---------------------------------------------------------------------------
// shared-memory tile C2C node (any smooth n <= kMaxOnChip, any strides)
// ---------------------------------------------------------------------------
static int tile_max_threads(int maxe) { return maxe <= 16 ? 512 : 256; }

// threads needed so every stage fits the per-thread butterfly budget
static int tile_threads(int n, const std::vector<int>& radices, int c, int maxe) {
  int need = 32;
  for (int R : radices) {
    const int64_t bf = int64_t(c) * (n / R);
    const int per = maxe / R;
    need = std::max<int64_t>(need, (bf + per - 1) / per);
  }
  return (need + 31) / 32 * 32;
}

bool choose_tile(int64_t n, bool interleaved, TileChoice& tc) {
  if (n > kMaxOnChip || !is_smooth(n)) return false;
  tc.radices = factor_radices(n, 16);
  tc.ld = spad_len(int(n));
  for (int maxe : {16, 32}) {
    tc.maxe = maxe;
    int c = interleaved ? 16 : int(std::max<int64_t>(1, std::min<int64_t>(64, 4096 / n)));
    while (c > 1 && (tile_smem_bytes(tc.ld, c) > 160 * 1024 ||
                     tile_threads(int(n), tc.radices, c, maxe) > tile_max_threads(maxe)))
      c /= 2;
    if (tile_smem_bytes(tc.ld, c) <= 200 * 1024 &&
        tile_threads(int(n), tc.radices, c, maxe) <= tile_max_threads(maxe)) {
      tc.c = c;
      tc.nthr = std::max(64, tile_threads(int(n), tc.radices, c, maxe));
      return true;
    }
  }
  return false;
}

struct C2CTileNode : Node {
  TileLaunch base{};
  int maxe = 16, dir = -1;
  DevBuf tw;
  std::vector<int> radices;
  cudaError_t run(const void* in, void* out, void*, cudaStream_t st) const override {
    TileLaunch L = base;
    L.in = static_cast<const float2*>(in);
    L.out = static_cast<float2*>(out);
    return launch_c2c_tile(maxe, dir, L, st);
  }
  std::string describe() const override {
    std::ostringstream o;
    o << "(c2c-tile n=" << base.desc.n << " c=" << base.c << " threads=" << base.nthr
      << " radices=";
    for (size_t i = 0; i < radices.size(); ++i) o << (i ? "x" : "") << radices[i];
    o << ")";
    return o.str();
  }
};

static std::unique_ptr<C2CTileNode> make_tile(int64_t n, int64_t ntr, const Addr& ia, const Addr& oa,
                                              int dir, float scale, bool interleaved,
                                              std::string* why) {
  TileChoice tc;
  if (!choose_tile(n, interleaved, tc)) {
    if (why) *why = "no on-chip schedule for n=" + std::to_string(n);
    return nullptr;
  }
  auto node = std::make_unique<C2CTileNode>();
  std::vector<float2> tw;
  node->base.desc = make_desc(int(n), tc.radices, tw);
  if (node->tw.upload(tw) != cudaSuccess) {
    if (why) *why = "device allocation failed";
    return nullptr;
  }
  node->base.tw = node->tw.as<float2>();
  node->base.ntr = ntr;
  node->base.ia = ia;
  node->base.oa = oa;
  node->base.c = tc.c;
  node->base.nthr = tc.nthr;
  node->base.ld = tc.ld;
  node->base.scale = scale;
  node->base.post = TwoLevel{nullptr, nullptr, 0, 1};
  node->maxe = tc.maxe;
  node->dir = dir;
  node->radices = tc.radices;
  return node;
}

// ---------------------------------------------------------------------------
// four-step C2C node: n = n1 * n2, both on chip
//   pass 1: length-n1 column transforms over stride n2, times W_n^{n2 k1},
//           into scratch Y[k1][n2]
//   pass 2: length-n2 row transforms of Y, stored transposed to X[k1 + n1 k2]
// The batch is processed in chunks so the scratch stays near L2 size.
// ---------------------------------------------------------------------------
struct C2CFourStepNode : Node {
  int64_t n = 0, n1 = 0, n2 = 0;
  Layout lay{};
  int64_t chunk = 1;
  std::unique_ptr<C2CTileNode> p1, p2;
  DevBuf lo, hi;
  size_t workspace() const override { return size_t(chunk) * size_t(n) * sizeof(float2); }
  int launches() const override { return int(2 * ((lay.howmany + chunk - 1) / chunk)); }
  cudaError_t run(const void* in, void* out, void* ws, cudaStream_t st) const override {
    const float2* x = static_cast<const float2*>(in);
    float2* y = static_cast<float2*>(out);
    float2* s = static_cast<float2*>(ws);
    for (int64_t m0 = 0; m0 < lay.howmany; m0 += chunk) {
      const int64_t cnt = std::min(chunk, lay.howmany - m0);
      TileLaunch a = p1->base;
      a.in = x + m0 * lay.idist;
      a.out = s;
      a.ntr = cnt * n2;
      cudaError_t e = launch_c2c_tile(p1->maxe, p1->dir, a, st);
      if (e != cudaSuccess) return e;
      TileLaunch b = p2->base;
      b.in = s;
      b.out = y + m0 * lay.odist;
      b.ntr = cnt * n1;
      e = launch_c2c_tile(p2->maxe, p2->dir, b, st);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  std::string describe() const override {
    std::ostringstream o;
    o << "(c2c-four-step n=" << n << " " << n1 << "x" << n2 << " chunk=" << chunk << " "
      << p1->describe() << " " << p2->describe() << ")";
    return o.str();
  }
};

int64_t four_step_split(int64_t n) {
  // n1 <= n2, both smooth and on chip, n1 as close to sqrt(n) as possible
  int64_t best = 0;
  for (int64_t d = 2; d * d <= n; ++d) {
    if (n % d) continue;
    const int64_t e = n / d;
    if (d <= kMaxOnChip && e <= kMaxOnChip && is_smooth(d) && is_smooth(e)) best = d;
  }
  return best;
}

// power-of-two four-step: both passes are static register kernels
// (fourstep.cu); members are processed in chunks whose intermediate stays
// near L2 size.  Dense batches (unit strides, 16-byte aligned members) run
// the bulk-copy ring passes of fourstep_ring.cu instead.
struct C2CFourStepPow2Node : Node {
  int64_t n = 0, n1 = 0, n2 = 0, chunk = 1;
  int dir = -1;
  Layout lay{};
  FourStepLaunch p1{}, p2{};
  DevBuf tw1, tw2, lo, hi;
  // ring form: tile widths and slots of each pass (c1 = 0: not used)
  int c1 = 0, c2 = 0, slots1 = 3, slots2 = 3;
  HostWord status;
  void status_words(std::vector<int*>& out) const override { out.push_back(status.p); }
  size_t workspace() const override { return size_t(chunk) * size_t(n) * sizeof(float2); }
  int launches() const override { return int(2 * ((lay.howmany + chunk - 1) / chunk)); }
  bool ring_ok(const void* in, const void* out) const {
    return c1 > 0 && lay.istride == 1 && lay.ostride == 1 && lay.idist % 2 == 0 && lay.odist % 2 == 0 &&
           reinterpret_cast<uintptr_t>(in) % 16 == 0 && reinterpret_cast<uintptr_t>(out) % 16 == 0;
  }
  cudaError_t run(const void* in, void* out, void* ws, cudaStream_t st) const override {
    const float2* x = static_cast<const float2*>(in);
    float2* y = static_cast<float2*>(out);
    float2* s = static_cast<float2*>(ws);
    const bool ring = ring_ok(in, out) && reinterpret_cast<uintptr_t>(ws) % 16 == 0;
    for (int64_t m0 = 0; m0 < lay.howmany; m0 += chunk) {
      const int64_t cnt = std::min(chunk, lay.howmany - m0);
      cudaError_t e;
      if (ring) {
        const uint32_t r1 = uint32_t(std::min<int64_t>(n1, 256)), r2 = uint32_t(std::min<int64_t>(n2, 256));
        FourStepRingLaunch a{};
        FourStepRingLaunch b{};
        e = encode_tensor_map_c64(&a.tm_in, x + m0 * lay.idist, uint64_t(n2), uint64_t(n1), uint64_t(cnt),
                                  uint64_t(n2) * 8u, uint64_t(lay.idist) * 8u, uint32_t(c1), r1);
        if (e == cudaSuccess)
          e = encode_tensor_map_c64(&a.tm_out, s, uint64_t(n2), uint64_t(n1), uint64_t(cnt), uint64_t(n2) * 8u,
                                    uint64_t(n) * 8u, uint32_t(c1), r1);
        if (e == cudaSuccess)
          e = encode_tensor_map_c64(&b.tm_out, y + m0 * lay.odist, uint64_t(n1), uint64_t(n2), uint64_t(cnt),
                                    uint64_t(n1) * 8u, uint64_t(lay.odist) * 8u, uint32_t(c2), r2);
        if (e != cudaSuccess) return e;
        a.blocks = n2 / c1;
        a.tiles = cnt * a.blocks;
        a.slots = slots1;
        a.scale = 1.f;
        a.tw = p1.tw;
        a.post = p1.post;
        a.err = status.device();
        e = launch_fourstep_ring(int(n1), c1, dir, 0, a, st);
        if (e != cudaSuccess) return e;
        b.in = s;
        b.idist = n;
        b.blocks = n1 / c2;
        b.tiles = cnt * b.blocks;
        b.slots = slots2;
        b.scale = p2.scale;
        b.tw = p2.tw;
        b.post = TwoLevel{nullptr, nullptr, 0, 1};
        b.err = status.device();
        e = launch_fourstep_ring(int(n2), c2, dir, 1, b, st);
        if (e != cudaSuccess) return e;
        continue;
      }
      FourStepLaunch a = p1;
      a.in = x + m0 * lay.idist;
      a.out = s;
      a.count = cnt * n2;
      e = launch_fourstep_pass(int(n1), dir, a, st);
      if (e != cudaSuccess) return e;
      FourStepLaunch b = p2;
      b.in = s;
      b.out = y + m0 * lay.odist;
      b.count = cnt * n1;
      e = launch_fourstep_pass(int(n2), dir, b, st);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  std::string describe() const override {
    std::ostringstream o;
    o << "(c2c-four-step-pow2 n=" << n << " " << n1 << "x" << n2 << " chunk=" << chunk << " c=" << p1.c << "/"
      << p2.c;
    if (c1) o << " bulk-ring c=" << c1 << "/" << c2 << " slots=" << slots1 << "/" << slots2;
    o << ")";
    return o.str();
  }
};

// ring-pass shape for a sub-transform length and pass: tile width and slots
// (PLFFT_B200_FSR_C / _SLOTS override both passes, _C1 / _S1 and _C2 / _S2
// one pass), the slots reduced to fit
static bool fourstep_ring_shape(int nl, int pass, int& c, int& slots) {
  // measured best at 2^14..2^20: 8-column tiles; two slots (more CTAs per
  // SM) up to nl = 256, three above
  c = 8;
  slots = nl <= 256 ? 2 : 3;
  c = env_int("PLFFT_B200_FSR_C", c);
  slots = env_int("PLFFT_B200_FSR_SLOTS", slots);
  c = env_int(pass == 0 ? "PLFFT_B200_FSR_C1" : "PLFFT_B200_FSR_C2", c);
  slots = env_int(pass == 0 ? "PLFFT_B200_FSR_S1" : "PLFFT_B200_FSR_S2", slots);
  if (!fourstep_ring_supported(nl, c)) return false;
  while (slots > 2 && fourstep_ring_smem(nl, c, slots) > 220 * 1024) --slots;
  return slots >= 2 && fourstep_ring_smem(nl, c, slots) <= 220 * 1024;
}

static int fourstep_c(int nl) {
  const int t = nl / fourstep_pass_e(nl);
  int c = std::min(env_int("PLFFT_B200_FS_C", 8), std::max(1, 512 / t));
  while (c > 1 && fourstep_pass_smem(nl, c) > 200 * 1024) c /= 2;
  return c;
}

// ring_shape: {c1, slots1, c2, slots2} of the bulk-copy ring passes (all 0:
// the defaults); c_override selects the per-element passes with that width
static std::unique_ptr<Node> make_four_step_pow2(int64_t n, const Layout& lay, int dir, float scale,
                                                 int c_override = 0, int chunk_mb = 0,
                                                 const int* ring_shape = nullptr) {
  if (!is_pow2(n) || std::getenv("PLFFT_B200_NO_FS_POW2")) return nullptr;
  int b = ilog2(n);
  const int64_t n1 = int64_t(1) << (b / 2), n2 = n / n1;
  if (!fourstep_pass_supported(int(n1)) || !fourstep_pass_supported(int(n2))) return nullptr;
  auto node = std::make_unique<C2CFourStepPow2Node>();
  node->n = n;
  node->n1 = n1;
  node->n2 = n2;
  node->dir = dir;
  node->lay = lay;
  const int64_t target = int64_t(chunk_mb ? chunk_mb : env_int("PLFFT_B200_FS_CHUNK_MB", 512)) << 20;
  node->chunk = std::max<int64_t>(1, std::min<int64_t>(lay.howmany, target / (n * 8)));
  auto stage_table = [&](int64_t nl, DevBuf& buf) {
    const int e = fourstep_pass_e(int(nl));
    std::vector<int> radices;
    int64_t rest = nl;
    int ke = 0;
    while (rest % e == 0 && rest > 1) {
      rest /= e;
      ++ke;
    }
    if (rest > 1) radices.push_back(int(rest));
    for (int i = 0; i < ke; ++i) radices.push_back(e);
    std::vector<float2> tw;
    make_desc(int(nl), radices, tw);
    return buf.upload(tw) == cudaSuccess;
  };
  if (!stage_table(n1, node->tw1) || !stage_table(n2, node->tw2)) return nullptr;
  const int64_t L = int64_t(1) << ((ilog2(n) + 1) / 2);
  std::vector<float2> lo(L), hi((n + L - 1) / L);
  for (int64_t i = 0; i < L; ++i) lo[i] = root_f(i, n, -1);
  for (size_t i = 0; i < hi.size(); ++i) hi[i] = root_f(int64_t(i) * L, n, -1);
  if (node->lo.upload(lo) != cudaSuccess || node->hi.upload(hi) != cudaSuccess) return nullptr;
  // pass 1: sub-transform g = (member, column n2 index), element k = n1 index
  node->p1 = FourStepLaunch{nullptr, nullptr, 0, n2, lay.idist, lay.istride, n2 * lay.istride, n, 1, n2,
                            c_override ? c_override : fourstep_c(int(n1)), 1.0f, node->tw1.as<float2>(),
                            TwoLevel{node->lo.as<float2>(), node->hi.as<float2>(), n, int(L)}};
  // pass 2: sub-transform g = (member, row k1), element k = n2 index
  node->p2 = FourStepLaunch{nullptr, nullptr, 0, n1, n, n2, 1, lay.odist, lay.ostride, n1 * lay.ostride,
                            c_override ? c_override : fourstep_c(int(n2)), scale, node->tw2.as<float2>(),
                            TwoLevel{nullptr, nullptr, 0, 1}};
  if (node->status.alloc() != cudaSuccess) return nullptr;
  if (!std::getenv("PLFFT_B200_NO_FS_RING") && !c_override && lay.istride == 1 && lay.ostride == 1) {
    int c1, s1, c2, s2;
    bool ok = fourstep_ring_shape(int(n1), 0, c1, s1) && fourstep_ring_shape(int(n2), 1, c2, s2);
    if (ring_shape) {
      c1 = ring_shape[0];
      s1 = ring_shape[1];
      c2 = ring_shape[2];
      s2 = ring_shape[3];
      ok = fourstep_ring_supported(int(n1), c1) && fourstep_ring_supported(int(n2), c2) &&
           fourstep_ring_smem(int(n1), c1, s1) <= 220 * 1024 && fourstep_ring_smem(int(n2), c2, s2) <= 220 * 1024 &&
           s1 >= 2 && s2 >= 2 && s1 <= 4 && s2 <= 4;
      if (!ok) return nullptr;
    }
    if (ok && n2 % c1 == 0 && n1 % c2 == 0) {
      node->c1 = c1;
      node->c2 = c2;
      node->slots1 = s1;
      node->slots2 = s2;
    }
  }
  return node;
}

// single-pass four-step for n = 65536 on an 8-CTA cluster (fourstep_cluster.cu)
struct C2CFourStepClusterNode : Node {
  int dir = -1, clusters = 1;
  FourStepClusterLaunch base{};
  DevBuf tw, lo, hi;
  cudaError_t run(const void* in, void* out, void*, cudaStream_t st) const override {
    FourStepClusterLaunch L = base;
    L.in = static_cast<const float2*>(in);
    L.out = static_cast<float2*>(out);
    return launch_fourstep_cluster(dir, L, clusters, st);
  }
  std::string describe() const override {
    std::ostringstream o;
    o << "(c2c-four-step-cluster n=65536 256x256 one pass, 8-CTA clusters x" << clusters << ")";
    return o.str();
  }
};

static std::unique_ptr<Node> make_four_step_cluster(int64_t n, const Layout& lay, int dir, float scale) {
  if (n != 65536) return nullptr;
  const int cap = fourstep_cluster_capacity();
  if (cap < 1) return nullptr;
  auto node = std::make_unique<C2CFourStepClusterNode>();
  node->dir = dir;
  node->clusters = cap;
  std::vector<float2> tw;
  make_desc(256, std::vector<int>{16, 16}, tw);
  const int64_t L = 256;
  std::vector<float2> lo(L), hi(n / L);
  for (int64_t i = 0; i < L; ++i) lo[i] = root_f(i, n, -1);
  for (int64_t i = 0; i < n / L; ++i) hi[i] = root_f(i * L, n, -1);
  if (node->tw.upload(tw) != cudaSuccess || node->lo.upload(lo) != cudaSuccess ||
      node->hi.upload(hi) != cudaSuccess)
    return nullptr;
  node->base = FourStepClusterLaunch{nullptr, nullptr, lay.howmany, lay.istride, lay.idist, lay.ostride, lay.odist,
                                     scale, node->tw.as<float2>(),
                                     TwoLevel{node->lo.as<float2>(), node->hi.as<float2>(), n, int(L)}};
  return node;
}

static std::unique_ptr<Node> make_four_step(int64_t n, const Layout& lay, int dir, float scale,
                                            std::string* why) {
  const int64_t best = four_step_split(n);
  if (!best) {
    if (why) *why = "length " + std::to_string(n) + " has no on-chip four-step split";
    return nullptr;
  }
  auto node = std::make_unique<C2CFourStepNode>();
  node->n = n;
  node->n1 = best;
  node->n2 = n / best;
  node->lay = lay;
  const int64_t target = 48ll << 20;  // scratch bytes per chunk
  node->chunk = std::max<int64_t>(1, std::min<int64_t>(lay.howmany, target / (n * 8)));
  const int64_t n1 = node->n1, n2 = node->n2;
  // pass 1: transforms g = (member, column n2), element k = n1 index
  Addr ia1{lay.idist, lay.istride, n2 * lay.istride, n2};
  Addr oa1{n, 1, n2, n2};
  node->p1 = make_tile(n1, 0, ia1, oa1, dir, 1.0f, true, why);
  // pass 2: transforms g = (member, row k1), element k = n2 index
  Addr ia2{n, n2, 1, n1};
  Addr oa2{lay.odist, lay.ostride, n1 * lay.ostride, n1};
  node->p2 = make_tile(n2, 0, ia2, oa2, dir, scale, false, why);
  if (!node->p1 || !node->p2) return nullptr;
  // two-level twiddle tables for W_n^e, e < n: lo[e % L] * hi[e / L]
  int64_t L = int64_t(1) << ((ilog2(n) + 1) / 2);
  std::vector<float2> lo(L), hi((n + L - 1) / L);
  for (int64_t i = 0; i < L; ++i) lo[i] = root_f(i, n, -1);
  for (size_t i = 0; i < hi.size(); ++i) hi[i] = root_f(int64_t(i) * L, n, -1);
  if (node->lo.upload(lo) != cudaSuccess || node->hi.upload(hi) != cudaSuccess) {
    if (why) *why = "device allocation failed";
    return nullptr;
  }
  node->p1->base.post = TwoLevel{node->lo.as<float2>(), node->hi.as<float2>(), n, int(L)};
  return node;
}

// ---------------------------------------------------------------------------
// split-BF16 tensor-core precision (split_bf16.cu): n = 256 or 4096 in one
// pass, n = 256 x 256 and 256 x 4096 as a four-step pair of passes
// ---------------------------------------------------------------------------
static uint16_t bf16_rn(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  u += 0x7fffu + ((u >> 16) & 1u);  // round to nearest even (finite inputs)
  return uint16_t(u >> 16);
}
static double bf16_val(uint16_t h) {
  const uint32_t u = uint32_t(h) << 16;
  float f;
  std::memcpy(&f, &u, 4);
  return double(f);
}

// three bf16 splits of the real 32x32 form of the DFT-16 matrix
// exp(dir 2 pi i iq / 16), packed two columns per 32-bit word
static std::vector<uint32_t> split_dft16(int dir) {
  std::vector<uint32_t> out(3 * 32 * 16);
  for (int row = 0; row < 32; ++row)
    for (int col = 0; col < 32; ++col) {
      const int i = row & 15, q = col & 15;
      const double ang = double(dir) * 2.0 * M_PI * double((i * q) % 16) / 16.0;
      const double wr = std::cos(ang), wi = std::sin(ang);
      // [Re W, -Im W; Im W, Re W]
      const double a = row < 16 ? (col < 16 ? wr : -wi) : (col < 16 ? wi : wr);
      double r = a;
      for (int s = 0; s < 3; ++s) {
        const uint16_t h = bf16_rn(float(r));
        r -= bf16_val(h);
        uint32_t& w = out[size_t(s) * 512 + size_t(row) * 16 + size_t(col / 2)];
        w |= (col & 1) ? uint32_t(h) << 16 : uint32_t(h);
      }
    }
  return out;
}

struct SplitBf16Node : Node {
  int64_t n = 0, n1 = 0, n2 = 0, chunk = 1;  // n2 == 0: one pass of length n1
  int dir = -1;
  Layout lay{};
  FourStepLaunch p1{}, p2{};
  DevBuf tw1, tw2, lo, hi, dftm;
  size_t workspace() const override { return n2 ? size_t(chunk) * size_t(n) * sizeof(float2) : 0; }
  int launches() const override { return n2 ? int(2 * ((lay.howmany + chunk - 1) / chunk)) : 1; }
  cudaError_t run(const void* in, void* out, void* ws, cudaStream_t st) const override {
    const float2* x = static_cast<const float2*>(in);
    float2* y = static_cast<float2*>(out);
    const uint32_t* m = dftm.as<uint32_t>();
    if (!n2) {
      FourStepLaunch a = p1;
      a.in = x;
      a.out = y;
      return launch_split_bf16_pass(int(n1), dir, a, m, st);
    }
    float2* s = static_cast<float2*>(ws);
    for (int64_t m0 = 0; m0 < lay.howmany; m0 += chunk) {
      const int64_t cnt = std::min(chunk, lay.howmany - m0);
      FourStepLaunch a = p1;
      a.in = x + m0 * lay.idist;
      a.out = s;
      a.count = cnt * n2;
      cudaError_t e = launch_split_bf16_pass(int(n1), dir, a, m, st);
      if (e != cudaSuccess) return e;
      FourStepLaunch b = p2;
      b.in = s;
      b.out = y + m0 * lay.odist;
      b.count = cnt * n1;
      e = launch_split_bf16_pass(int(n2), dir, b, m, st);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  std::string describe() const override {
    std::ostringstream o;
    o << "(c2c-split-bf16 n=" << n << " radix-16 DFT-matrix stages on tensor cores, 3-term bf16 splits";
    if (n2) o << ", four-step " << n1 << "x" << n2 << " chunk=" << chunk;
    o << ")";
    return o.str();
  }
};

static std::unique_ptr<Node> make_split_bf16(int64_t n, const Layout& lay, int dir, float scale, std::string* why) {
  auto node = std::make_unique<SplitBf16Node>();
  node->n = n;
  node->dir = dir;
  node->lay = lay;
  if (n == 256 || n == 4096) {
    node->n1 = n;
  } else if (n == 65536 || n == (int64_t(1) << 20)) {
    node->n1 = 256;
    node->n2 = n / 256;
  } else {
    if (why) *why = "split-BF16 precision covers n = 256, 4096, 65536 and 2^20";
    return nullptr;
  }
  auto stage_table = [&](int64_t nl, DevBuf& buf) {
    std::vector<int> radices(nl == 256 ? 2 : 3, 16);
    std::vector<float2> tw;
    make_desc(int(nl), radices, tw);
    return buf.upload(tw) == cudaSuccess;
  };
  const std::vector<uint32_t> mat = split_dft16(dir);
  if (node->dftm.upload(mat) != cudaSuccess || !stage_table(node->n1, node->tw1) ||
      (node->n2 && !stage_table(node->n2, node->tw2))) {
    if (why) *why = "device allocation failed";
    return nullptr;
  }
  const int64_t n1 = node->n1, n2 = node->n2;
  if (!n2) {
    node->p1 = FourStepLaunch{nullptr, nullptr, lay.howmany, 1, lay.idist, 0, lay.istride, lay.odist, 0,
                              lay.ostride, split_bf16_pass_c(int(n1)), scale, node->tw1.as<float2>(),
                              TwoLevel{nullptr, nullptr, 0, 1}};
    return node;
  }
  const int64_t target = int64_t(env_int("PLFFT_B200_FS_CHUNK_MB", 512)) << 20;
  node->chunk = std::max<int64_t>(1, std::min<int64_t>(lay.howmany, target / (n * 8)));
  const int64_t L = int64_t(1) << ((ilog2(n) + 1) / 2);
  std::vector<float2> lo(L), hi((n + L - 1) / L);
  for (int64_t i = 0; i < L; ++i) lo[i] = root_f(i, n, -1);
  for (size_t i = 0; i < hi.size(); ++i) hi[i] = root_f(int64_t(i) * L, n, -1);
  if (node->lo.upload(lo) != cudaSuccess || node->hi.upload(hi) != cudaSuccess) {
    if (why) *why = "device allocation failed";
    return nullptr;
  }
  // pass 1: columns (member, n2 index), element k = n1 index, times W_n^{col k}
  node->p1 = FourStepLaunch{nullptr, nullptr, 0, n2, lay.idist, lay.istride, n2 * lay.istride, n, 1, n2,
                            split_bf16_pass_c(int(n1)), 1.0f, node->tw1.as<float2>(),
                            TwoLevel{node->lo.as<float2>(), node->hi.as<float2>(), n, int(L)}};
  // pass 2: rows (member, n1 index), element k = n2 index, written transposed
  node->p2 = FourStepLaunch{nullptr, nullptr, 0, n1, n, n2, 1, lay.odist, lay.ostride, n1 * lay.ostride,
                            split_bf16_pass_c(int(n2)), scale, node->tw2.as<float2>(), TwoLevel{nullptr, nullptr, 0, 1}};
  return node;
}

std::unique_ptr<Node> make_c2c_node(int64_t n, const Layout& lay, int dir, float scale,
                                    int precision, std::string* why) {
  if (precision == 1) return make_split_bf16(n, lay, dir, scale, why);
  const bool unit = lay.istride == 1 && lay.ostride == 1;
  const bool interleaved = !unit && (lay.howmany > 1) &&
                           (std::llabs(lay.idist) < lay.istride || std::llabs(lay.odist) < lay.ostride);
  if (unit && !std::getenv("PLFFT_B200_NO_POW2")) {
    auto p2 = make_pow2(n, lay, dir, scale, why);
    if (p2) return p2;
  }
  RegChoice rc;
  if (unit && choose_reg(n, rc)) {
    auto node = std::make_unique<C2CRegNode>();
    std::vector<float2> tw;
    node->base.desc = make_desc(int(n), rc.radices, tw);
    if (node->tw.upload(tw) != cudaSuccess) {
      if (why) *why = "device allocation failed";
      return nullptr;
    }
    node->base.tw = node->tw.as<float2>();
    node->base.howmany = lay.howmany;
    node->base.istride = lay.istride;
    node->base.idist = lay.idist;
    node->base.ostride = lay.ostride;
    node->base.odist = lay.odist;
    node->base.t = rc.t;
    node->base.g = rc.g;
    node->base.scale = scale;
    node->e = rc.e;
    node->dir = dir;
    node->radices = rc.radices;
    return node;
  }
  if (n <= kMaxOnChip && is_smooth(n)) {
    Addr ia{lay.idist, 0, lay.istride, 1};
    Addr oa{lay.odist, 0, lay.ostride, 1};
    auto t = make_tile(n, lay.howmany, ia, oa, dir, scale, interleaved, why);
    if (t) return t;
  }
  if (std::getenv("PLFFT_B200_CLUSTER"))
    if (auto fc = make_four_step_cluster(n, lay, dir, scale)) return fc;
  if (auto fs = make_four_step_pow2(n, lay, dir, scale)) return fs;
  if (is_smooth(n)) return make_four_step(n, lay, dir, scale, why);
  return make_conv_node(n, lay, dir, scale, why);
}

// Alternative schedules for the same C2C problem, default first (the
// autotuner times them).  level 1: launch shapes of the chosen kernel
// family; level 2: also other kernel families and radix sizes; level 3:
// also four-step CTA shapes and chunk sizes.
std::vector<std::unique_ptr<Node>> make_c2c_candidates(int64_t n, const Layout& lay, int dir, float scale,
                                                       int precision, int level) {
  std::vector<std::unique_ptr<Node>> out;
  std::string why;
  if (auto d = make_c2c_node(n, lay, dir, scale, precision, &why)) out.push_back(std::move(d));
  if (precision != 0 || out.empty()) return out;
  const bool unit = lay.istride == 1 && lay.ostride == 1;
  if (unit && is_pow2(n) && n >= 64 && n <= 8192) {
    std::vector<int> es{pow2_default_e(n)};
    if (level >= 2)
      for (int e : {16, 32})
        if (e != es[0] && pow2_supported(int(n), e)) es.push_back(e);
    for (int e : es) {
      const int t = int(n / e);
      for (int ring : {0, 1, 3}) {
        for (int g : {1, 2, 4, 8}) {
          if (ring == 3 && g != 1) continue;  // warp-group rings size themselves
          if (g * t > (e <= 16 ? 512 : 256)) continue;
          Pow2Params pp;
          pp.e = e;
          pp.ring = ring;
          pp.g = g;
          if (auto c = make_pow2(n, lay, dir, scale, &why, pp)) out.push_back(std::move(c));
        }
      }
    }
  }
  if (level >= 2 && n <= kMaxOnChip && is_smooth(n)) {
    const bool interleaved = !unit && (lay.howmany > 1) &&
                             (std::llabs(lay.idist) < lay.istride || std::llabs(lay.odist) < lay.ostride);
    Addr ia{lay.idist, 0, lay.istride, 1};
    Addr oa{lay.odist, 0, lay.ostride, 1};
    if (auto t = make_tile(n, lay.howmany, ia, oa, dir, scale, interleaved, &why)) out.push_back(std::move(t));
  }
  if (!is_smooth(n) && conv_fused_length(n)) {
    // shapes of the one-launch convolution kernel, and members per CTA
    const int64_t m = conv_fused_length(n);
    for (const auto& sh : conv_fused_shapes(int(m))) {
      const int t = int(m / sh.first);
      const int gdef = std::max(1, 64 / t);
      for (int g : {gdef, 2 * gdef, gdef / 2}) {
        if (g < 1 || g * t > std::max(256, t) || (g != gdef && level < 2)) continue;
        if (auto c = make_conv_fused(n, lay, dir, scale, &why, sh.first, sh.second, g)) out.push_back(std::move(c));
      }
    }
  }
  if (is_pow2(n) && n > 8192) {
    // the one-pass cluster form (one HBM round trip, but latency-bound at
    // 8 warps per SM: 1.13 TB/s against 1.8 for two passes at 2^16 x 1024)
    if (level >= 2)
      if (auto f = make_four_step_cluster(n, lay, dir, scale)) out.push_back(std::move(f));
    for (int c : {4, 8, 16})
      for (int mb : {128, 512, 1024}) {
        if (level < 3 && mb != 512) continue;
        if (auto f = make_four_step_pow2(n, lay, dir, scale, c, mb)) out.push_back(std::move(f));
      }
    // shapes of the bulk-copy ring passes (dense batches)
    if (unit) {
      const int64_t n1 = int64_t(1) << (ilog2(n) / 2), n2 = n / n1;
      auto shapes = [](int64_t nl) {
        return nl <= 512 ? std::vector<std::pair<int, int>>{{8, 2}, {8, 3}, {16, 3}}
                         : std::vector<std::pair<int, int>>{{8, 3}, {4, 2}, {4, 3}};
      };
      for (const auto& a : shapes(n1))
        for (const auto& b : shapes(n2)) {
          const int rs[4] = {a.first, a.second, b.first, b.second};
          if (auto f = make_four_step_pow2(n, lay, dir, scale, 0, 0, rs)) out.push_back(std::move(f));
        }
    }
  }
  // drop duplicates of the default (same description)
  std::vector<std::unique_ptr<Node>> uniq;
  for (auto& c : out) {
    bool dup = false;
    for (auto& u : uniq) dup = dup || u->describe() == c->describe();
    if (!dup) uniq.push_back(std::move(c));
  }
  return uniq;
}

plfft_status_t take_device_status(const Node* node) {
  if (!node) return PLFFT_OK;
  std::vector<int*> words;
  node->status_words(words);
  plfft_status_t st = PLFFT_OK;
  for (int* w : words) {
    if (w && *reinterpret_cast<volatile int*>(w) != 0) {
      st = PLFFT_DEVICE_TIMEOUT;
      *reinterpret_cast<volatile int*>(w) = 0;
    }
  }
  return st;
}

PlanData::~PlanData() {
  if (stream) cudaStreamDestroy(stream);
  for (auto& st : pipe_st)
    if (st) cudaStreamDestroy(st);
  for (auto& row : pipe_ev)
    for (auto& ev : row)
      if (ev) cudaEventDestroy(ev);
}

}  // namespace plfft_b200
