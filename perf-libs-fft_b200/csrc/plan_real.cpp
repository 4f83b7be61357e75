// Plan nodes for R2C, C2R and R2R built on a C2C plan (realwrap.cu).
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <sstream>

#include "plan.hpp"

namespace plfft_b200 {

namespace {

struct RealWrapNode : Node {
  int kind = 0;
  int64_t n = 0, len = 0, nout = 0;
  Layout lay{};
  double scale = 1.0;
  int wmode_in = AW_NONE, wmode_out = AW_NONE;
  bool fp64 = false;
  int64_t chunk = 1;
  size_t cbytes() const { return fp64 ? sizeof(double2) : sizeof(float2); }
  std::unique_ptr<Node> inner;  // C2C of length len over `chunk` contiguous members, in place
  void status_words(std::vector<int*>& out) const override { inner->status_words(out); }
  size_t inner_ws() const { return inner->workspace(); }
  size_t workspace() const override {
    const size_t work = size_t(chunk) * size_t(len) * cbytes();
    return ((work + 255) & ~size_t(255)) + inner_ws();
  }
  int launches() const override {
    const int64_t chunks = (lay.howmany + chunk - 1) / chunk;
    return int(chunks * (2 + inner->launches()));
  }
  cudaError_t run(const void* in, void* out, void* ws, cudaStream_t st) const override {
    void* work = ws;
    const size_t work_bytes = (size_t(chunk) * size_t(len) * cbytes() + 255) & ~size_t(255);
    void* iws = static_cast<char*>(ws) + work_bytes;
    RealWrapLaunch L{in,        out,       work,     n,          len,        nout, lay.istride, lay.idist, lay.ostride,
                     lay.odist, scale,     wmode_in, wmode_out, fp64 ? 1 : 0};
    for (int64_t m0 = 0; m0 < lay.howmany; m0 += chunk) {
      const int64_t cnt = std::min(chunk, lay.howmany - m0);
      cudaError_t e = launch_realwrap(true, kind, L, m0, cnt, st);
      if (e != cudaSuccess) return e;
      e = run_inner(cnt, work, iws, st);
      if (e != cudaSuccess) return e;
      e = launch_realwrap(false, kind, L, m0, cnt, st);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  // the inner plan was built for `chunk` members; the last chunk may be
  // shorter, which only changes which members hold meaningful data
  cudaError_t run_inner(int64_t, void* work, void* iws, cudaStream_t st) const {
    return inner->run(work, work, iws, st);
  }
  std::string describe() const override {
    static const char* names[] = {"r2c", "c2r", "dct1", "dct2", "dct3", "dct4", "dst1",
                                  "dst2", "dst3", "dst4", "dht", "r2hc", "hc2r"};
    std::ostringstream o;
    o << "(" << names[kind] << (fp64 ? "-fp64" : "") << "-via-c2c n=" << n << " len=" << len << " chunk=" << chunk << " "
      << inner->describe() << ")";
    return o.str();
  }
};

int64_t wrap_len(int kind, int64_t n) {
  switch (kind) {
    case RW_DCT1: return 2 * (n - 1);
    case RW_DST1: return 2 * (n + 1);
    case RW_DCT2:
    case RW_DCT3:
    case RW_DCT4:
    case RW_DST2:
    case RW_DST3:
    case RW_DST4: return 2 * n;
    default: return n;
  }
}

int wrap_dir(int kind) {
  switch (kind) {
    case RW_C2R:
    case RW_HC2R:
    case RW_DCT3:
    case RW_DST3: return +1;
    default: return -1;
  }
}

// R2C / C2R of even n = 2m through a length-m C2C over the real data read as
// complex pairs (realwrap.cu, launch_real_half): R2C = C2C in place of the
// user's input into work, then the split; C2R = the merge into work, then the
// C2C into the user's output.  Members whose real side is not 8-byte aligned
// (odd real distance or base) run the generic full-length node instead.
struct RealHalfNode : Node {
  bool r2c = true;
  int64_t n = 0, m = 0, chunk = 1;
  Layout lay{};
  float scale = 1.f;
  int wmode_in = AW_NONE, wmode_out = AW_NONE;
  DevBuf tw;
  std::unique_ptr<Node> inner, inner_last;  // `chunk` members, and the last chunk's remainder
  std::unique_ptr<Node> generic;
  void status_words(std::vector<int*>& out) const override {
    inner->status_words(out);
    if (inner_last) inner_last->status_words(out);
    generic->status_words(out);
  }
  size_t work_bytes() const { return (size_t(chunk) * size_t(m) * sizeof(float2) + 255) & ~size_t(255); }
  size_t workspace() const override {
    size_t iw = inner->workspace();
    if (inner_last) iw = std::max(iw, inner_last->workspace());
    return std::max(work_bytes() + iw, generic->workspace());
  }
  int launches() const override {
    const int64_t chunks = (lay.howmany + chunk - 1) / chunk;
    return int(chunks * (1 + inner->launches()));
  }
  bool paired(const void* real_side, int64_t real_dist) const {
    return reinterpret_cast<uintptr_t>(real_side) % 8 == 0 && (lay.howmany == 1 || real_dist % 2 == 0);
  }
  cudaError_t run(const void* in, void* out, void* ws, cudaStream_t st) const override {
    if (r2c ? !paired(in, lay.idist) : !paired(out, lay.odist)) return generic->run(in, out, ws, st);
    float2* work = static_cast<float2*>(ws);
    void* iws = static_cast<char*>(ws) + work_bytes();
    RealHalfLaunch L{};
    L.work = work;
    L.m = m;
    L.istride = lay.istride;
    L.idist = lay.idist;
    L.ostride = lay.ostride;
    L.odist = lay.odist;
    L.scale = scale;
    L.wmode_in = wmode_in;
    L.wmode_out = wmode_out;
    L.tw = tw.as<float2>();
    for (int64_t m0 = 0; m0 < lay.howmany; m0 += chunk) {
      const int64_t cnt = std::min(chunk, lay.howmany - m0);
      const Node& c2c = (cnt < chunk && inner_last) ? *inner_last : *inner;
      cudaError_t e;
      if (r2c) {
        const float2* z = static_cast<const float2*>(in) + m0 * (lay.idist / 2);
        L.out = static_cast<float2*>(out);
        e = c2c.run(z, work, iws, st);
        if (e == cudaSuccess) e = launch_real_half(true, L, m0, cnt, st);
      } else {
        L.in = static_cast<const float2*>(in);
        e = launch_real_half(false, L, m0, cnt, st);
        if (e == cudaSuccess) e = c2c.run(work, static_cast<float2*>(out) + m0 * (lay.odist / 2), iws, st);
      }
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  std::string describe() const override {
    std::ostringstream o;
    o << "(" << (r2c ? "r2c" : "c2r") << "-half n=" << n << " m=" << m << " chunk=" << chunk << " "
      << inner->describe() << ")";
    return o.str();
  }
};

}  // namespace

static std::unique_ptr<Node> make_realwrap_generic(int kind, int64_t n, const Layout& lay, double scale,
                                                   std::string* why, int wmode_in, int wmode_out, bool fp64);

std::unique_ptr<Node> make_realwrap_node(int kind, int64_t n, const Layout& lay, double scale, std::string* why,
                                         int wmode_in, int wmode_out, bool fp64) {
  // FP32 R2C / C2R of even n with unit real stride: the half-length form
  const bool half = (kind == RW_R2C || kind == RW_C2R) && !fp64 && n >= 4 && n % 2 == 0 &&
                    (kind == RW_R2C ? lay.istride == 1 : lay.ostride == 1) &&
                    (kind == RW_R2C ? lay.idist >= n : lay.odist >= n) &&
                    (kind == RW_R2C ? wmode_in == AW_NONE : wmode_out == AW_NONE) &&
                    !std::getenv("PLFFT_B200_NO_REAL_HALF");
  if (!half) return make_realwrap_generic(kind, n, lay, scale, why, wmode_in, wmode_out, fp64);
  auto node = std::make_unique<RealHalfNode>();
  node->r2c = kind == RW_R2C;
  node->n = n;
  node->m = n / 2;
  node->lay = lay;
  node->scale = float(scale);
  node->wmode_in = wmode_in;
  node->wmode_out = wmode_out;
  node->generic = make_realwrap_generic(kind, n, lay, scale, why, wmode_in, wmode_out, false);
  if (!node->generic) return nullptr;
  const int64_t m = node->m;
  const int64_t target = 64ll << 20;  // bytes of complex work per chunk
  node->chunk = std::max<int64_t>(1, std::min<int64_t>(lay.howmany, target / (m * int64_t(sizeof(float2)))));
  auto inner_for = [&](int64_t count) {
    // R2C: pairs of the input (complex distance idist / 2) into work; C2R:
    // work into pairs of the output (odist / 2), with the plan's scale
    return node->r2c ? make_c2c_node(m, Layout{count, 1, lay.idist / 2, 1, m}, -1, 1.0f, 0, why)
                     : make_c2c_node(m, Layout{count, 1, m, 1, lay.odist / 2}, +1, float(scale), 0, why);
  };
  node->inner = inner_for(node->chunk);
  if (!node->inner) return nullptr;
  const int64_t rem = lay.howmany % node->chunk;
  if (rem) {
    node->inner_last = inner_for(rem);
    if (!node->inner_last) return nullptr;
  }
  std::vector<float2> tw(size_t(m) + 1);
  for (int64_t k = 0; k <= m; ++k) {  // W_n^k
    double c, sn;
    unit_root(k, n, c, sn);
    tw[k] = make_float2(float(c), float(-sn));
  }
  if (node->tw.upload(tw) != cudaSuccess) {
    if (why) *why = "device allocation failed";
    return nullptr;
  }
  return node;
}

static std::unique_ptr<Node> make_realwrap_generic(int kind, int64_t n, const Layout& lay, double scale,
                                                   std::string* why, int wmode_in, int wmode_out, bool fp64) {
  if (kind == RW_DCT1 && n < 2) {
    if (why) *why = "DCT-I needs n > 1";
    return nullptr;
  }
  auto node = std::make_unique<RealWrapNode>();
  node->kind = kind;
  node->n = n;
  node->len = wrap_len(kind, n);
  node->nout = kind == RW_R2C ? n / 2 + 1 : n;
  node->lay = lay;
  node->scale = scale;
  node->wmode_in = wmode_in;
  node->wmode_out = wmode_out;
  node->fp64 = fp64;
  const int64_t target = 64ll << 20;  // bytes of complex work per chunk
  node->chunk = std::max<int64_t>(1, std::min<int64_t>(lay.howmany, target / (node->len * int64_t(node->cbytes()))));
  Layout inner{node->chunk, 1, node->len, 1, node->len};
  node->inner = fp64 ? make_fp64_c2c(node->len, inner, wrap_dir(kind), 1.0, why)
                     : make_c2c_node(node->len, inner, wrap_dir(kind), 1.0f, 0, why);
  if (!node->inner) return nullptr;
  return node;
}

}  // namespace plfft_b200

namespace plfft_b200 {

namespace {

// One-kernel R2C / C2R / DCT-II..IV / DST-II..IV / R2HC / HC2R / DHT for
// N = 2M, M a power of two (real_fused.cu); unit element stride.
struct RealFusedNode : Node {
  int kind = 0, m = 0;
  RealFusedLaunch base{};
  DevBuf tab;
  cudaError_t run(const void* in, void* out, void*, cudaStream_t st) const override {
    RealFusedLaunch L = base;
    L.in = in;
    L.out = out;
    const bool in_real = kind != FR_C2R, out_real = kind != FR_R2C;
    L.pairs_in = in_real && (reinterpret_cast<uintptr_t>(in) % 8 == 0) && (L.howmany == 1 || L.idist % 2 == 0);
    L.pairs_out = out_real && (reinterpret_cast<uintptr_t>(out) % 8 == 0) && (L.howmany == 1 || L.odist % 2 == 0);
    L.quads_in = in_real && (reinterpret_cast<uintptr_t>(in) % 16 == 0) && (L.howmany == 1 || L.idist % 4 == 0);
    return launch_real_fused(kind, m, L, st);
  }
  std::string describe() const override {
    static const char* names[] = {"r2c", "c2r",  "dct2", "dst2", "dct3", "dst3",
                                  "dct4", "dst4", "r2hc", "hc2r", "dht"};
    std::ostringstream o;
    o << "(" << names[kind] << "-fused n=" << 2 * m << " m=" << m << " e=" << base.e << " g=" << base.g
      << ")";
    return o.str();
  }
};

}  // namespace

std::unique_ptr<Node> make_real_fused_node(int kind, int64_t n, const Layout& lay, float scale, int wmode, int g_override,
                                           int e_override) {
  if (n % 2 || !real_fused_supported(int(n / 2)) || lay.istride != 1 || lay.ostride != 1) return nullptr;
  if (std::getenv("PLFFT_B200_NO_FUSED_REAL")) return nullptr;
  const int m = int(n / 2);
  int e = real_fused_e(m);
  if (const char* v = std::getenv("PLFFT_B200_RF_E"))  // launch-shape experiments
    if (m == 512 && std::atoi(v) == 32) e = 32;
  if (e_override && (e_override == e || (m == 512 && e_override == 32))) e = e_override;
  std::vector<int> radices;
  int rest = m, ke = 0;
  while (rest % e == 0 && rest > 1) {
    rest /= e;
    ++ke;
  }
  if (rest > 1) radices.push_back(rest);
  for (int i = 0; i < ke; ++i) radices.push_back(e);
  std::vector<float2> tw;
  make_desc(m, radices, tw);
  const bool iv = kind == FR_DCT4 || kind == FR_DST4;
  const size_t post_off = tw.size();
  for (int k = 0; k <= m; ++k) {  // W_N^k; DCT-IV / DST-IV: exp(i pi k / N) = W_{2N}^{-k}
    double c, s;
    unit_root(iv ? 2 * int64_t(k) : k, iv ? 4 * n : n, c, s);
    tw.push_back(make_float2(float(c), float(iv ? s : -s)));
  }
  const size_t rot_off = tw.size();
  for (int k = 0; k <= m; ++k) {  // exp(-i pi k / 2N) = W_{4N}^k; DCT-IV / DST-IV: exp(i pi (4k+1) / 4N)
    double c, s;
    unit_root(iv ? 4 * int64_t(k) + 1 : k, iv ? 8 * n : 4 * n, c, s);
    tw.push_back(make_float2(float(c), float(iv ? s : -s)));
  }
  auto node = std::make_unique<RealFusedNode>();
  node->kind = kind;
  node->m = m;
  if (node->tab.upload(tw) != cudaSuccess) return nullptr;
  const int t = m / e;
  node->base.howmany = lay.howmany;
  node->base.idist = lay.idist;
  node->base.odist = lay.odist;
  node->base.g = std::max(1, 128 / t);
  if (const char* v = std::getenv("PLFFT_B200_RF_G")) node->base.g = std::max(1, std::atoi(v));
  if (g_override) node->base.g = g_override;
  if (t * node->base.g > 1024) return nullptr;
  node->base.g = std::max(node->base.g, std::max(1, 32 / t));  // whole warps (the kernel shuffles)
  node->base.e = e;
  node->base.wmode = wmode;
  node->base.scale = scale;
  node->base.tw = node->tab.as<float2>();
  node->base.post = node->tab.as<float2>() + post_off;
  node->base.rot = node->tab.as<float2>() + rot_off;
  return node;
}

}  // namespace plfft_b200

namespace plfft_b200 {

// Alternative schedules of a real-data transform for the autotuner, the
// default first: the fused kernel with other transforms-per-CTA counts and
// (N = 1024) the other register split, then the three-launch real-wrap
// schedule around a C2C.
std::vector<std::unique_ptr<Node>> make_real_candidates(int fused_kind, int wrap_kind, int64_t n, const Layout& lay,
                                                        float scale, int level) {
  std::vector<std::unique_ptr<Node>> out;
  std::string why;
  auto fused = fused_kind >= 0 ? make_real_fused_node(fused_kind, n, lay, scale) : nullptr;
  if (fused) {
    const int g0 = static_cast<RealFusedNode*>(fused.get())->base.g;
    const int e0 = static_cast<RealFusedNode*>(fused.get())->base.e;
    out.push_back(std::move(fused));
    for (int g : {g0 / 2, g0 * 2, g0 / 4, g0 * 4}) {
      if (g < 1 || g == g0) continue;
      if (auto c = make_real_fused_node(fused_kind, n, lay, scale, 0, g)) out.push_back(std::move(c));
    }
    if (n == 1024) {
      for (int g : {g0, g0 / 2, g0 * 2})
        if (g >= 1)
          if (auto c = make_real_fused_node(fused_kind, n, lay, scale, 0, g, e0 == 16 ? 32 : 16)) out.push_back(std::move(c));
    }
  }
  if (out.empty() || level >= 2) {
    if (auto w = make_realwrap_node(wrap_kind, n, lay, scale, &why)) out.push_back(std::move(w));
  }
  // keep the first of schedules that describe alike
  std::vector<std::unique_ptr<Node>> uniq;
  for (auto& c : out) {
    bool dup = false;
    for (auto& u : uniq) dup = dup || u->describe() == c->describe();
    if (!dup) uniq.push_back(std::move(c));
  }
  return uniq;
}

}  // namespace plfft_b200
