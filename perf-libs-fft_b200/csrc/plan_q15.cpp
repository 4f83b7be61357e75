// Q0.15 fixed-point C2C plan node (kernels in q15.cu).
//
// The reference plans fixed-point C2C / R2C / C2R and rejects fixed-point
// R2R (src/plfft.cpp:248-261); every fixed-point transform is scaled by
// 1/n (docs/plfft.md:128-130).  The device path covers C2C of power-of-two
// n <= 256 with the reference's ESTIMATE decomposition; other fixed-point
// configurations fail plan creation with a reason.
#include <cmath>

#include "plan.hpp"

namespace plfft_b200 {

// sat16(trunc(float(x) * 2^15)) (reference src/plfft_convert.hpp:48-54)
static int16_t cvt_q15(double x) {
  const float f = float(x) * 32768.0f;
  const double t = std::trunc(double(f));
  return int16_t(t > 32767.0 ? 32767 : (t < -32768.0 ? -32768 : int(t)));
}

static int pack16(int16_t lo, int16_t hi) { return int(uint16_t(lo)) | (int(hi) << 16); }

struct Q15Node : Node {
  int n = 0, dir = -1;
  Q15Launch base{};
  DevBuf tw;
  cudaError_t run(const void* in, void* out, void*, cudaStream_t st) const override {
    Q15Launch L = base;
    L.in = static_cast<const int*>(in);
    L.out = static_cast<int*>(out);
    return launch_q15(n, dir, L, st);
  }
  std::string describe() const override {
    return "(c2c-q15 n=" + std::to_string(n) + (n <= 16 ? " one codelet" : " 16-column x twiddled-row codelets") +
           ")";
  }
};

std::unique_ptr<Node> make_q15_node(int64_t n, const Layout& lay, int dir, std::string* why) {
  if (!q15_supported(n)) {
    if (why) *why = "fixed-point C2C on the device covers power-of-two n <= 256";
    return nullptr;
  }
  auto node = std::make_unique<Q15Node>();
  node->n = int(n);
  node->dir = dir;
  node->base.howmany = lay.howmany;
  node->base.istride = lay.istride;
  node->base.idist = lay.idist;
  node->base.ostride = lay.ostride;
  node->base.odist = lay.odist;
  if (n >= 32) {
    // row twiddles (reference src/generate_twiddles.hpp:72-132, n1 = n/16,
    // n2 = 16, premultiplied pairs)
    const int64_t m = n / 16;
    std::vector<int2> w;
    const double base = double(dir) * 2.0 * M_PI / double(n);
    for (int64_t j = 1; j < m; ++j)
      for (int64_t i = 1; i < 16; ++i) {
        const double ang = base * double(i) * double(j);
        const double a = std::cos(ang), b = std::sin(ang);
        w.push_back(make_int2(pack16(cvt_q15(a), cvt_q15(b)), pack16(cvt_q15(-b), cvt_q15(a))));
      }
    if (node->tw.upload(w) != cudaSuccess) {
      if (why) *why = "device allocation failed";
      return nullptr;
    }
    node->base.tw = node->tw.as<int2>();
  }
  return node;
}

}  // namespace plfft_b200
