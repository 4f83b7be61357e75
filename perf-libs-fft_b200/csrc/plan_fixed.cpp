// Fixed-point plan node, Q0.15 and Q0.7 (kernels in fixed_point.cu).
//
// The reference plans fixed-point C2C / R2C / C2R and rejects fixed-point
// R2R (src/plfft.cpp:248-261); every fixed-point transform is scaled by
// 1/n (docs/plfft.md:128-130).  The device path covers C2C, R2C and C2R of
// power-of-two n <= 4096 with the reference's ESTIMATE decomposition
// (radix-16 cooley_tukey_ab, over a radix-16 cooley_tukey_ac for n > 256;
// the R2C levels with mirrored rows, the C2R ones decimating in frequency
// over the Hermitian half); other fixed-point configurations fail plan
// creation with a reason.
#include <cmath>

#include "plan.hpp"

namespace plfft_b200 {

// sat(trunc(float(x) * 2^(bits-1))) (reference src/plfft_convert.hpp:36-54)
static short cvt_fixed(double x, int bits) {
  const float f = float(x) * float(1 << (bits - 1));
  const double t = std::trunc(double(f));
  const double hi = double((1 << (bits - 1)) - 1), lo = -double(1 << (bits - 1));
  return short(t > hi ? hi : (t < lo ? lo : t));
}

// premultiplied twiddles of a radix-16 level over n1 rows (reference
// src/generate_twiddles.hpp:72-132 with n2 = 16): for j = 1..n1-1,
// i = 1..15, angle dir 2 pi i j / (16 n1): (c, s, cvt(-s), c)
static std::vector<short4> radix16_twiddles(int64_t n1, int dir, int bits) {
  std::vector<short4> w;
  const double base = double(dir) * 2.0 * M_PI / double(16 * n1);
  for (int64_t j = 1; j < n1; ++j)
    for (int64_t i = 1; i < 16; ++i) {
      const double ang = base * double(i) * double(j);
      const double a = std::cos(ang), b = std::sin(ang);
      w.push_back(make_short4(cvt_fixed(a, bits), cvt_fixed(b, bits), cvt_fixed(-b, bits), cvt_fixed(a, bits)));
    }
  return w;
}

struct FixedNode : Node {
  int bits = 16, n = 0, dir = -1;
  int kind = 0;  // 0 C2C, 1 R2C, 2 C2R
  FixedLaunch base{};
  DevBuf tw, tw2;
  cudaError_t run(const void* in, void* out, void*, cudaStream_t st) const override {
    FixedLaunch L = base;
    L.in = in;
    L.out = out;
    if (kind == 1) return launch_fixed_r2c(bits, n, L, st);
    if (kind == 2) return launch_fixed_c2r(bits, n, L, st);
    return launch_fixed(bits, n, dir, L, st);
  }
  std::string describe() const override {
    const char* shape = n <= 16 ? " one codelet" : (n <= 256 ? " 16-column x twiddled-row codelets"
                                                              : " 256-column codelets, radix-16 ac and ab levels");
    static const char* names[] = {"(c2c-", "(r2c-", "(c2r-"};
    static const char* notes[] = {"", ", mirrored rows", ", DIF rows of the Hermitian half"};
    return std::string(names[kind]) + (bits == 16 ? "q15" : "q7") + " n=" + std::to_string(n) + shape + notes[kind] +
           ")";
  }
};

// kind: 0 C2C (dir as given), 1 R2C (forward; input reals, output bins
// 0..n/2), 2 C2R (backward; input bins 0..n/2, output reals)
std::unique_ptr<Node> make_fixed_node(int bits, int64_t n, const Layout& lay, int dir, std::string* why, int kind) {
  if (!fixed_supported(n) || (kind != 0 && n < 2)) {
    if (why) *why = "fixed-point transforms on the device cover power-of-two n <= 4096 (R2C / C2R: n >= 2)";
    return nullptr;
  }
  if (n > 256 && lay.howmany > 0x7fffffffLL) {
    if (why) *why = "fixed-point n > 256 takes one CTA per member: batch too large";
    return nullptr;
  }
  auto node = std::make_unique<FixedNode>();
  node->bits = bits;
  node->n = int(n);
  node->kind = kind;
  node->dir = kind == 1 ? -1 : (kind == 2 ? 1 : dir);
  dir = node->dir;
  node->base.howmany = lay.howmany;
  node->base.istride = lay.istride;
  node->base.idist = lay.idist;
  node->base.ostride = lay.ostride;
  node->base.odist = lay.odist;
  if (n >= 32) {
    if (node->tw.upload(radix16_twiddles(n / 16, dir, bits)) != cudaSuccess) {
      if (why) *why = "device allocation failed";
      return nullptr;
    }
    node->base.tw = node->tw.as<short4>();
  }
  if (n >= 512) {
    if (node->tw2.upload(radix16_twiddles(n / 256, dir, bits)) != cudaSuccess) {
      if (why) *why = "device allocation failed";
      return nullptr;
    }
    node->base.tw2 = node->tw2.as<short4>();
  }
  return node;
}

}  // namespace plfft_b200
