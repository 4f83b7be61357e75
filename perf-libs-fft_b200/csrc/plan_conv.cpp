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

std::unique_ptr<Node> make_conv_node(int64_t n, const Layout& lay, int dir, float scale, std::string* why) {
  auto node = std::make_unique<ConvNode>();
  node->dir = dir;
  node->n = n;
  node->lay = lay;
  node->scale = scale;
  node->rader = is_prime(n) && is_smooth(n - 1) && n > 2;
  node->m = node->rader ? n - 1 : next_smooth(2 * n - 1);
  const int64_t m = node->m;
  const int64_t target = 64ll << 20;
  node->chunk = std::max<int64_t>(1, std::min<int64_t>(lay.howmany, target / (m * 8)));
  Layout inner{node->chunk, 1, m, 1, m};
  node->fwd = make_c2c_node(m, inner, -1, 1.0f, 0, why);
  node->bwd = make_c2c_node(m, inner, +1, 1.0f, 0, why);
  if (!node->fwd || !node->bwd) return nullptr;

  std::vector<cd> b(m, cd(0, 0));
  if (node->rader) {
    const int64_t g = primitive_root(n);
    const int64_t ginv = pow_mod(g, n - 2, n);
    std::vector<int> pin(m), pout(m);
    int64_t gq = 1, gi = 1;
    for (int64_t q = 0; q < m; ++q) {
      pin[q] = int(gq);
      pout[q] = int(gi);
      double c, s;
      unit_root(gi, n, c, s);  // b_q = exp(dir 2 pi i g^-q / P)
      b[q] = cd(c, dir * s);
      gq = gq * g % n;
      gi = gi * ginv % n;
    }
    if (node->pin.upload(pin) != cudaSuccess || node->pout.upload(pout) != cudaSuccess) {
      if (why) *why = "device allocation failed";
      return nullptr;
    }
  } else {
    // w_k = exp(dir i pi (k^2 mod 2n) / n); b_m = conj(w_m), wrapped
    std::vector<cd> w(n);
    for (int64_t k = 0; k < n; ++k) {
      const int64_t e = int64_t((__int128)k * k % (2 * n));
      double c, s;
      unit_root(e, 2 * n, c, s);
      w[k] = cd(c, dir * s);
    }
    for (int64_t k = 0; k < n; ++k) {
      b[k] = std::conj(w[k]);
      if (k) b[m - k] = std::conj(w[k]);
    }
    if (node->chirp.upload(to_f2(w, 1.0)) != cudaSuccess) {
      if (why) *why = "device allocation failed";
      return nullptr;
    }
  }
  const std::vector<cd> B = host_fft(b, -1);
  if (node->spec.upload(to_f2(B, 1.0 / double(m))) != cudaSuccess) {
    if (why) *why = "device allocation failed";
    return nullptr;
  }
  return node;
}

}  // namespace plfft_b200
