// FP64 plan nodes (kernels in fp64.cu).
//
// C2C: one shared-memory pass for 7-smooth n <= 4096 (radices 8, 7, 5, 4,
// 3, 2), direct sums for other n <= 4096, a two-pass four-step for
// 7-smooth n = n1 n2 with both factors <= 4096.  R2C / C2R: the real data
// widened into a length-n complex sequence (Hermitian expansion for C2R),
// the C2C plan, then the half spectrum (or the real parts) extracted.
// Every table is computed in double on the host.
#include <cmath>
#include <sstream>

#include "plan.hpp"

namespace plfft_b200 {

namespace {

constexpr int kF64MaxOnChip = 4096;

bool smooth7(int64_t n) {
  for (int p : {2, 3, 5, 7})
    while (n % p == 0) n /= p;
  return n == 1;
}

std::vector<int> f64_radices(int64_t n) {
  std::vector<int> r;
  for (int p : {8, 7, 5, 4, 3, 2})
    while (n % p == 0) {
      r.push_back(p);
      n /= p;
    }
  return r;
}

double2 root64(int64_t k, int64_t n) {  // exp(-2 pi i k / n)
  double c, s;
  unit_root(k, n, c, s);
  return make_double2(c, -s);
}

struct F64Tables {
  DevBuf tw, omega;
  F64Desc desc{};
  bool build(int n, bool direct) {
    desc = F64Desc{};
    desc.n = n;
    std::vector<double2> tw_h, om_h;
    if (direct) {
      for (int m = 0; m < n; ++m) tw_h.push_back(root64(m, n));
      om_h.push_back(make_double2(1.0, 0.0));
    } else {
      const std::vector<int> rad = f64_radices(n);
      if (rad.size() > 24) return false;
      int ns = 1;
      for (size_t s = 0; s < rad.size(); ++s) {
        const int R = rad[s];
        F64Stage& st = desc.st[s];
        st.radix = R;
        st.ns = ns;
        st.tw_off = int(tw_h.size());
        st.om_off = int(om_h.size());
        if (ns > 1)
          for (int i = 1; i < R; ++i)
            for (int r = 0; r < ns; ++r) tw_h.push_back(root64(int64_t(r) * i, int64_t(ns) * R));
        for (int q = 0; q < R; ++q) om_h.push_back(root64(q, R));
        ns *= R;
      }
      desc.nstages = int(rad.size());
      if (tw_h.empty()) tw_h.push_back(make_double2(1.0, 0.0));
    }
    return tw.upload(tw_h) == cudaSuccess && omega.upload(om_h) == cudaSuccess;
  }
};

struct F64C2CNode : Node {
  int64_t n = 0, n1 = 0, n2 = 0, chunk = 1;  // n2 == 0: one pass of length n
  int dir = -1;
  bool direct = false;
  Layout lay{};
  double scale = 1.0;
  F64Tables t1, t2;
  DevBuf lo, hi;
  size_t workspace() const override { return n2 ? size_t(chunk * n) * sizeof(double2) : 0; }
  int launches() const override { return n2 ? int(2 * ((lay.howmany + chunk - 1) / chunk)) : 1; }
  F64TileLaunch pass(const F64Tables& t, const void* in, void* out, int64_t ntr, Addr ia, Addr oa, double sc,
                     TwoLevel64 post) const {
    return F64TileLaunch{static_cast<const double2*>(in), static_cast<double2*>(out), ntr, ia, oa, sc, t.desc,
                         t.tw.as<double2>(), t.omega.as<double2>(), post};
  }
  cudaError_t run(const void* in, void* out, void* ws, cudaStream_t st) const override {
    const TwoLevel64 none{nullptr, nullptr, 0, 1};
    if (!n2) {
      Addr ia{lay.idist, 0, lay.istride, 1}, oa{lay.odist, 0, lay.ostride, 1};
      return launch_fp64_tile(dir, direct, pass(t1, in, out, lay.howmany, ia, oa, scale, none), st);
    }
    const auto* x = static_cast<const double2*>(in);
    auto* y = static_cast<double2*>(out);
    auto* s = static_cast<double2*>(ws);
    const TwoLevel64 tw2{lo.as<double2>(), hi.as<double2>(), n, int64_t(std::ceil(std::sqrt(double(n))))};
    for (int64_t m0 = 0; m0 < lay.howmany; m0 += chunk) {
      const int64_t cnt = std::min(chunk, lay.howmany - m0);
      // pass 1: columns (member, n2 index) of length n1, times W_n^{col k}
      Addr ia1{lay.idist, lay.istride, n2 * lay.istride, n2}, oa1{n, 1, n2, n2};
      cudaError_t e = launch_fp64_tile(dir, false, pass(t1, x + m0 * lay.idist, s, cnt * n2, ia1, oa1, 1.0, tw2), st);
      if (e != cudaSuccess) return e;
      // pass 2: rows (member, n1 index) of length n2, written transposed
      Addr ia2{n, n2, 1, n1}, oa2{lay.odist, lay.ostride, n1 * lay.ostride, n1};
      e = launch_fp64_tile(dir, false, pass(t2, s, y + m0 * lay.odist, cnt * n1, ia2, oa2, scale, none), st);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  std::string describe() const override {
    std::ostringstream o;
    o << "(c2c-fp64 n=" << n;
    if (n2)
      o << " four-step " << n1 << "x" << n2 << " chunk=" << chunk;
    else
      o << (direct ? " direct sums" : " shared-memory Stockham");
    o << ")";
    return o.str();
  }
};

struct F64RealNode : Node {
  std::unique_ptr<Node> c2c;  // length-n complex plan over a dense chunk
  F64RealLaunch base{};
  int64_t howmany = 1, chunk = 1;
  size_t work_bytes() const { return size_t(chunk * base.n) * sizeof(double2); }
  size_t workspace() const override { return (work_bytes() + 255) / 256 * 256 + c2c->workspace(); }
  int launches() const override { return int((howmany + chunk - 1) / chunk) * (2 + c2c->launches()); }
  cudaError_t run(const void* in, void* out, void* ws, cudaStream_t st) const override {
    F64RealLaunch L = base;
    L.in = in;
    L.out = out;
    L.work = static_cast<double2*>(ws);
    void* cws = static_cast<unsigned char*>(ws) + (work_bytes() + 255) / 256 * 256;
    for (int64_t m0 = 0; m0 < howmany; m0 += chunk) {
      const int64_t cnt = std::min(chunk, howmany - m0);
      if (cnt != chunk) return cudaErrorInvalidValue;  // chunk divides the batch (see make_fp64_node)
      cudaError_t e = launch_fp64_real(true, L, m0, cnt, st);
      if (e == cudaSuccess) e = c2c->run(L.work, L.work, cws, st);
      if (e == cudaSuccess) e = launch_fp64_real(false, L, m0, cnt, st);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  std::string describe() const override {
    return std::string(base.c2r ? "(c2r" : "(r2c") + "-fp64 through complex n=" + std::to_string(base.n) + ") + " +
           c2c->describe();
  }
};

}  // namespace

std::unique_ptr<Node> make_fp64_c2c(int64_t n, const Layout& lay, int dir, double scale, std::string* why) {
  auto node = std::make_unique<F64C2CNode>();
  node->n = n;
  node->dir = dir;
  node->lay = lay;
  node->scale = scale;
  if (n <= kF64MaxOnChip) {
    node->direct = !smooth7(n);
    if (!node->t1.build(int(n), node->direct)) return nullptr;
    return node;
  }
  if (!smooth7(n)) {
    if (why) *why = "FP64 on the device covers 7-smooth n, and other n <= 4096";
    return nullptr;
  }
  // four-step split with both factors on chip, n1 as close to sqrt(n) as possible
  int64_t best = 0;
  for (int64_t a = 2; a <= kF64MaxOnChip; ++a)
    if (n % a == 0 && n / a <= kF64MaxOnChip && (!best || std::llabs(a * a - n) < std::llabs(best * best - n))) best = a;
  if (!best) {
    if (why) *why = "FP64 length has no four-step split with factors <= 4096";
    return nullptr;
  }
  node->n1 = best;
  node->n2 = n / best;
  node->chunk = std::max<int64_t>(1, std::min<int64_t>(lay.howmany, (int64_t(256) << 20) / (n * 16)));
  if (!node->t1.build(int(node->n1), false) || !node->t2.build(int(node->n2), false)) return nullptr;
  const int64_t L = int64_t(std::ceil(std::sqrt(double(n))));
  std::vector<double2> lo(L), hi((n + L - 1) / L);
  for (int64_t i = 0; i < L; ++i) lo[i] = root64(i, n);
  for (size_t i = 0; i < hi.size(); ++i) hi[i] = root64(int64_t(i) * L, n);
  if (node->lo.upload(lo) != cudaSuccess || node->hi.upload(hi) != cudaSuccess) return nullptr;
  return node;
}

std::unique_ptr<Node> make_fp64_node(int kind, int64_t n, const Layout& lay, int dir, double scale,
                                     std::string* why) {
  if (kind == 0) return make_fp64_c2c(n, lay, dir, scale, why);
  if (kind != 1 && kind != 2) {
    if (why) *why = "FP64 real-to-real transforms have no device schedule";
    return nullptr;
  }
  auto node = std::make_unique<F64RealNode>();
  node->howmany = lay.howmany;
  // a chunk that divides the batch, of at most ~128 MB of complex workspace
  int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(lay.howmany, (int64_t(128) << 20) / (n * 16)));
  while (lay.howmany % chunk) --chunk;
  node->chunk = chunk;
  node->base = F64RealLaunch{nullptr, nullptr, nullptr, n, lay.istride, lay.idist, lay.ostride, lay.odist,
                             kind == 2 ? 1 : 0, scale};
  node->c2c = make_fp64_c2c(n, Layout{chunk, 1, n, 1, n}, kind == 2 ? 1 : -1, 1.0, why);
  if (!node->c2c) return nullptr;
  return node;
}

}  // namespace plfft_b200
