// Rader and Bluestein plan nodes, their FP64 host tables, and the strategy
// choice for lengths with prime factors above 13.
//
// Strategy order follows the reference planner (src/planner/planner.cpp:
// 49-182; rader before bluestein, rader_strategy fails when P-1 needs a
// convolution itself, src/planner/strategies/rader.hpp:816-856): prime P
// with smooth P-1 -> Rader; every other non-smooth length -> Bluestein with
// M = the smallest smooth length >= 2N-1 (src/factorize.hpp:74-87,
// src/planner/strategies/bluestein.hpp:721-779).
#include <algorithm>
#include <cmath>
#include <complex>
#include <sstream>

#include "plan.hpp"

namespace plfft_b200 {


// FP64 host FFT for smooth lengths (tables only): recursive decimation in
// time, each prime factor by a direct DFT, twiddles from an exact-index root
// table.
static void host_fft_rec(const cd* x, int64_t xs, cd* y, int64_t n, int sign, const std::vector<cd>& w, int64_t big,
                         std::vector<cd>& scratch, size_t off) {
  if (n == 1) {
    y[0] = x[0];
    return;
  }
  int64_t p = 2;
  while (n % p) ++p;
  const int64_t m = n / p;
  cd* sub = scratch.data() + off;
  for (int64_t r = 0; r < p; ++r) host_fft_rec(x + r * xs, xs * p, sub + r * m, m, sign, w, big, scratch, off + n);
  const int64_t step = big / n;
  std::vector<cd> t(p);
  for (int64_t k = 0; k < m; ++k) {
    for (int64_t r = 0; r < p; ++r) t[r] = sub[r * m + k] * w[(r * k * step) % big];
    for (int64_t q = 0; q < p; ++q) {
      cd acc = 0;
      for (int64_t r = 0; r < p; ++r) acc += t[r] * w[((r * q) % p) * (big / p)];
      y[k + m * q] = acc;
    }
  }
}

std::vector<cd> host_fft(const std::vector<cd>& x, int sign) {
  const int64_t n = int64_t(x.size());
  std::vector<cd> w(n), y(n);
  for (int64_t k = 0; k < n; ++k) {
    double c, s;
    unit_root(k, n, c, s);
    w[k] = cd(c, sign * s);
  }
  std::vector<cd> scratch(size_t(4 * n + 64));
  host_fft_rec(x.data(), 1, y.data(), n, sign, w, n, scratch, 0);
  return y;
}

std::vector<float2> to_f2(const std::vector<cd>& v, double scale) {
  std::vector<float2> r(v.size());
  for (size_t i = 0; i < v.size(); ++i) r[i] = make_float2(float(v[i].real() * scale), float(v[i].imag() * scale));
  return r;
}

int64_t pow_mod(int64_t a, int64_t e, int64_t p) {
  __int128 r = 1, b = a % p;
  while (e) {
    if (e & 1) r = (r * b) % p;
    b = (b * b) % p;
    e >>= 1;
  }
  return int64_t(r);
}

// smallest primitive root of prime p: g^((p-1)/q) != 1 for every prime q | p-1
int64_t primitive_root(int64_t p) {
  std::vector<int64_t> qs;
  int64_t m = p - 1;
  for (int64_t q = 2; q * q <= m; ++q)
    if (m % q == 0) {
      qs.push_back(q);
      while (m % q == 0) m /= q;
    }
  if (m > 1) qs.push_back(m);
  for (int64_t g = 2; g < p; ++g) {
    bool ok = true;
    for (int64_t q : qs)
      if (pow_mod(g, (p - 1) / q, p) == 1) {
        ok = false;
        break;
      }
    if (ok) return g;
  }
  return 1;
}

// smallest smooth length >= n (all factors on chip-capable radices), with a
// preference for lengths whose C2C plan is a single on-chip pass
int64_t next_smooth(int64_t n) {
  for (int64_t m = std::max<int64_t>(n, 1);; ++m)
    if (is_smooth(m)) return m;
}

namespace {

struct ConvNode : Node {
  bool rader = false;
  int dir = -1;
  int64_t n = 0, m = 0;
  Layout lay{};
  float scale = 1.f;
  int64_t chunk = 1;
  DevBuf chirp, spec, pin, pout;
  std::unique_ptr<Node> fwd, bwd;  // length-m C2C plans over `chunk` contiguous members, in place
  void status_words(std::vector<int*>& out) const override {
    fwd->status_words(out);
    bwd->status_words(out);
  }

  size_t work_bytes() const { return (size_t(chunk) * size_t(m) * sizeof(float2) + 255) & ~size_t(255); }
  size_t sum_bytes() const { return (size_t(chunk) * sizeof(float2) + 255) & ~size_t(255); }
  size_t workspace() const override {
    return work_bytes() + sum_bytes() + std::max(fwd->workspace(), bwd->workspace());
  }
  int launches() const override {
    const int64_t chunks = (lay.howmany + chunk - 1) / chunk;
    return int(chunks * (3 + fwd->launches() + bwd->launches()));
  }
  cudaError_t run(const void* in, void* out, void* ws, cudaStream_t st) const override {
    char* base = static_cast<char*>(ws);
    float2* work = reinterpret_cast<float2*>(base);
    float2* sum0 = reinterpret_cast<float2*>(base + work_bytes());
    void* iws = base + work_bytes() + sum_bytes();
    ConvLaunch L{};
    L.in = static_cast<const float2*>(in);
    L.out = static_cast<float2*>(out);
    L.work = work;
    L.sum0 = sum0;
    L.chirp = chirp.as<float2>();
    L.spec = spec.as<float2>();
    L.perm_in = pin.as<int>();
    L.perm_out = pout.as<int>();
    L.n = n;
    L.m = m;
    L.istride = lay.istride;
    L.idist = lay.idist;
    L.ostride = lay.ostride;
    L.odist = lay.odist;
    L.scale = scale;
    for (int64_t m0 = 0; m0 < lay.howmany; m0 += chunk) {
      const int64_t cnt = std::min(chunk, lay.howmany - m0);
      cudaError_t e = launch_conv(rader ? CONV_RD_PRE : CONV_BS_PRE, L, m0, cnt, st);
      if (e == cudaSuccess) e = fwd->run(work, work, iws, st);
      if (e == cudaSuccess) e = launch_conv(rader ? CONV_MUL_SAVE0 : CONV_MUL, L, m0, cnt, st);
      if (e == cudaSuccess) e = bwd->run(work, work, iws, st);
      if (e == cudaSuccess) e = launch_conv(rader ? CONV_RD_POST : CONV_BS_POST, L, m0, cnt, st);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  std::string describe() const override {
    std::ostringstream o;
    o << "(" << (rader ? "rader" : "bluestein") << " n=" << n << " m=" << m << " chunk=" << chunk << " "
      << fwd->describe() << ")";
    return o.str();
  }
};

}  // namespace

// Convolution tables.  Bluestein: w_k = exp(dir i pi (k^2 mod 2n) / n).
static std::vector<cd> bluestein_chirp(int64_t n, int dir) {
  std::vector<cd> w(n);
  for (int64_t k = 0; k < n; ++k) {
    const int64_t e = int64_t((__int128)k * k % (2 * n));
    double c, s;
    unit_root(e, 2 * n, c, s);
    w[k] = cd(c, dir * s);
  }
  return w;
}

// b_m = conj(w_|m|) for |m| < n, placed cyclically in a length-m sequence
// (m >= 2n - 1)
static std::vector<cd> bluestein_kernel(const std::vector<cd>& w, int64_t m) {
  const int64_t n = int64_t(w.size());
  std::vector<cd> b(m, cd(0, 0));
  for (int64_t k = 0; k < n; ++k) {
    b[k] = std::conj(w[k]);
    if (k) b[m - k] = std::conj(w[k]);
  }
  return b;
}

// Rader for prime p with generator g, l = p - 1: perm_in[q] = g^q,
// perm_out[q] = g^-q, and b_q = exp(dir 2 pi i g^-q / p) laid out for a
// length-m cyclic convolution (m = l exactly, or m >= 2l - 1 with the
// negative lags b_{l-j} at m - j so a zero-padded input convolves cyclically
// modulo l)
static void rader_tables(int64_t p, int dir, int64_t m, std::vector<int>& pin, std::vector<int>& pout,
                         std::vector<cd>& b) {
  const int64_t l = p - 1;
  const int64_t g = primitive_root(p);
  const int64_t ginv = pow_mod(g, p - 2, p);
  pin.assign(size_t(l), 0);
  pout.assign(size_t(l), 0);
  std::vector<cd> bl(l);
  int64_t gq = 1, gi = 1;
  for (int64_t q = 0; q < l; ++q) {
    pin[q] = int(gq);
    pout[q] = int(gi);
    double c, s;
    unit_root(gi, p, c, s);
    bl[q] = cd(c, dir * s);
    gq = gq * g % p;
    gi = gi * ginv % p;
  }
  b.assign(size_t(m), cd(0, 0));
  for (int64_t j = 0; j < l; ++j) b[j] = bl[j];
  for (int64_t j = 1; j < l; ++j) b[m - j] = bl[l - j];
}

namespace {

// One launch per execution: conv_fused_kernel over power-of-two m.
struct ConvFusedNode : Node {
  bool rader = false;
  int64_t n = 0, m = 0;
  Layout lay{};
  float scale = 1.f;
  int e = 16, minb = 3, g = 1;
  DevBuf tw, chirp, spec, pin, pout;
  cudaError_t run(const void* in, void* out, void*, cudaStream_t st) const override {
    ConvFusedLaunch L{};
    L.in = static_cast<const float2*>(in);
    L.out = static_cast<float2*>(out);
    L.howmany = lay.howmany;
    L.istride = lay.istride;
    L.idist = lay.idist;
    L.ostride = lay.ostride;
    L.odist = lay.odist;
    L.n = int(n);
    L.g = g;
    L.tw = tw.as<float2>();
    L.chirp = chirp.as<float2>();
    L.spec = spec.as<float2>();
    L.perm_in = pin.as<int>();
    L.perm_out = pout.as<int>();
    L.scale = scale;
    return launch_conv_fused(int(m), e, minb, rader, L, st);
  }
  std::string describe() const override {
    std::ostringstream o;
    o << "(" << (rader ? "rader" : "bluestein") << "-fused n=" << n << " m=" << m << " e=" << e << " minb=" << minb
      << " g=" << g << ")";
    return o.str();
  }
};

int64_t next_pow2(int64_t v) {
  int64_t p = 1;
  while (p < v) p <<= 1;
  return p;
}

}  // namespace

// the reference planner's choice (src/planner/planner.cpp:49-182,
// src/planner/strategies/rader.hpp:816-856): Rader for a prime whose p - 1
// needs no convolution itself, Bluestein for every other non-smooth length
static bool use_rader(int64_t n) { return n > 2 && is_prime(n) && is_smooth(n - 1); }

int64_t conv_fused_length(int64_t n) {
  if (n < 3) return 0;
  // Rader convolves l = n - 1 terms, Bluestein n: a cyclic length >= 2l - 1
  const int64_t m = next_pow2(std::max<int64_t>(64, use_rader(n) ? 2 * n - 3 : 2 * n - 1));
  return m <= 8192 ? m : 0;
}

// e = 0: the default shape for the length (PLFFT_B200_CONV_E / _MINB / _G
// override it), else the given shape
std::unique_ptr<Node> make_conv_fused(int64_t n, const Layout& lay, int dir, float scale, std::string* why, int e_req,
                                      int minb_req, int g_req) {
  if (std::getenv("PLFFT_B200_CONV_UNFUSED")) return nullptr;
  const int64_t m = conv_fused_length(n);
  if (m == 0) return nullptr;
  const bool rader = use_rader(n);
  const auto shapes = conv_fused_shapes(int(m));
  if (shapes.empty()) return nullptr;
  int e = shapes[0].first, minb = shapes[0].second;
  if (e_req) {
    e = e_req;
    minb = minb_req;
  } else {
    if (const char* v = std::getenv("PLFFT_B200_CONV_E")) e = std::atoi(v);
    if (const char* v = std::getenv("PLFFT_B200_CONV_MINB")) minb = std::atoi(v);
    if (!conv_fused_supported(int(m), e, minb))
      for (const auto& sh : shapes)
        if (sh.first == e) {
          minb = sh.second;
          break;
        }
  }
  if (!conv_fused_supported(int(m), e, minb)) {
    if (e_req) return nullptr;
    e = shapes[0].first;
    minb = shapes[0].second;
  }
  auto node = std::make_unique<ConvFusedNode>();
  node->rader = rader;
  node->n = n;
  node->m = m;
  node->lay = lay;
  node->scale = scale;
  node->e = e;
  node->minb = minb;
  const int t = int(m / e);
  const int maxthr = t > 256 ? t : 256;
  int g = std::max(1, 64 / t);
  if (g_req > 0)
    g = g_req;
  else if (const char* v = std::getenv("PLFFT_B200_CONV_G"))
    g = std::max(1, std::atoi(v));
  while (g > 1 && (g * t > maxthr || conv_fused_smem_bytes(int(m), g) > 160 * 1024)) g /= 2;
  node->g = g;
  // radices: leftover factor first, then radix-e stages (the order of the
  // compile-time stage list)
  std::vector<int> radices;
  int64_t rest = m;
  int ke = 0;
  while (rest % e == 0 && rest > 1) {
    rest /= e;
    ++ke;
  }
  if (rest > 1) radices.push_back(int(rest));
  for (int i = 0; i < ke; ++i) radices.push_back(e);
  std::vector<float2> tw;
  make_desc(int(m), radices, tw);
  std::vector<cd> b;
  cudaError_t err = node->tw.upload(tw);
  if (rader) {
    std::vector<int> pin, pout;
    rader_tables(n, dir, m, pin, pout, b);
    if (err == cudaSuccess) err = node->pin.upload(pin);
    if (err == cudaSuccess) err = node->pout.upload(pout);
  } else {
    const std::vector<cd> w = bluestein_chirp(n, dir);
    b = bluestein_kernel(w, m);
    if (err == cudaSuccess) err = node->chirp.upload(to_f2(w, 1.0));
  }
  if (err == cudaSuccess) err = node->spec.upload(to_f2(host_fft(b, -1), 1.0 / double(m)));
  if (err != cudaSuccess) {
    if (why) *why = "device allocation failed";
    return nullptr;
  }
  return node;
}

// Strategy (the reference planner's rule): Rader for prime n with smooth
// n - 1, else Bluestein.  Lengths whose convolution fits a power-of-two
// m <= 8192 run as one fused launch; longer ones convolve over m = n - 1
// (Rader) or the smallest smooth m >= 2n - 1 (Bluestein) with multi-launch
// length-m C2C plans.
std::unique_ptr<Node> make_conv_node(int64_t n, const Layout& lay, int dir, float scale, std::string* why) {
  if (auto f = make_conv_fused(n, lay, dir, scale, why, 0, 0, 0)) return f;
  auto node = std::make_unique<ConvNode>();
  node->dir = dir;
  node->n = n;
  node->lay = lay;
  node->scale = scale;
  node->rader = use_rader(n);
  node->m = node->rader ? n - 1 : next_smooth(2 * n - 1);
  const int64_t m = node->m;
  const int64_t target = 64ll << 20;
  node->chunk = std::max<int64_t>(1, std::min<int64_t>(lay.howmany, target / (m * 8)));
  Layout inner{node->chunk, 1, m, 1, m};
  node->fwd = make_c2c_node(m, inner, -1, 1.0f, 0, why);
  node->bwd = make_c2c_node(m, inner, +1, 1.0f, 0, why);
  if (!node->fwd || !node->bwd) return nullptr;

  std::vector<cd> b;
  cudaError_t err = cudaSuccess;
  if (node->rader) {
    std::vector<int> pin, pout;
    rader_tables(n, dir, m, pin, pout, b);
    err = node->pin.upload(pin);
    if (err == cudaSuccess) err = node->pout.upload(pout);
  } else {
    const std::vector<cd> w = bluestein_chirp(n, dir);
    b = bluestein_kernel(w, m);
    err = node->chirp.upload(to_f2(w, 1.0));
  }
  if (err == cudaSuccess) err = node->spec.upload(to_f2(host_fft(b, -1), 1.0 / double(m)));
  if (err != cudaSuccess) {
    if (why) *why = "device allocation failed";
    return nullptr;
  }
  return node;
}

}  // namespace plfft_b200
