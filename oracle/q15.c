/*
 * Bit-exact CPU restatement of the reference's Q0.15 C2C path --
 * TEST INFRASTRUCTURE ONLY (same rules as oracle.c: only tests/ and the
 * CPU-baseline leg of bench.py load it, to check results).
 *
 * What is restated (arm/perf-libs-fft):
 *   Arithmetic semantics (src/providers/jit/print_algo.cpp:1228-1230,
 *   src/providers/jit/emit.hpp:150-175 and :370-425, constant lowering
 *   print_algo.cpp:2150-2290):
 *     - every codelet input is pre-scaled by a rounding shift right by
 *       log2(radix) (srshr), so a whole transform is scaled by 1/N;
 *     - additions and subtractions saturate to int16 (sqadd / sqsub);
 *     - a multiply by a real constant k is (2 a k + 2^15) >> 16, saturated
 *       (sqrdmulh); multiplying by +-i swaps re/im and uses k = -32768 or
 *       32767 on the two lanes;
 *     - a complex product with a twiddle is two int16 x int16 products
 *       accumulated in 32 bits (smull / smlal / smlsl, wrapping) and
 *       narrowed once by a rounding, saturating shift by 15 (sqrshrn #15).
 *   Codelets: radix 2, 4, 8 and the fixed-point split-radix 16
 *   (src/providers/jit/split_radix_z16.cpp, selected for fixed point by
 *   src/providers/jit/wfta_nfact.cpp:89-97); the backward codelet of
 *   length r produces, at output k, the forward codelet's output r-k.
 *   Composition for N <= 16: one codelet per member.  For N = 16 m
 *   (m = 2, 4, 8, 16): stage 1 runs the length-m codelet down each of the
 *   16 columns x[c + 16 q]; stage 2 runs, for each row j of that result,
 *   a 16-point codelet whose inputs i >= 1 are first multiplied by the
 *   twiddle W_N^{dir i j} (row 0 untwiddled), writing y[j + m k]
 *   (the Cooley-Tukey "ab" level, src/planner/strategies/cooley_tukey.hpp:
 *   622-748, with the twiddled DIT codelet of asm/neon/
 *   plfft_ab_q15_jjjt_dit_gu.S).
 *   Twiddles: cvt(x) = sat16(trunc(float(x) * 2^15)) of cos and sin of
 *   dir*2*pi*i*j/N (src/generate_twiddles.hpp:72-132,
 *   src/plfft_convert.hpp:48-54).
 *
 * Parity pin: tests/golden/q15_reference.npz holds outputs of the
 * reference's own NEON kernels (executed from their source text by
 * tests/golden/neon_q15.py); tests/test_q15.py requires this file to match
 * them bit for bit.
 *
 * Data: interleaved int16 (re, im), members idist/odist complex elements
 * apart, unit element stride.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int32_t re, im;
} q15c;

static int32_t sat16(int64_t v) { return v > 32767 ? 32767 : (v < -32768 ? -32768 : (int32_t)v); }
static int32_t rshr(int32_t v, int s) { return (v + (1 << (s - 1))) >> s; }
/* sqrdmulh by a constant */
static int32_t rdm(int32_t a, int32_t k) { return sat16(((int64_t)2 * a * k + (1 << 15)) >> 16); }
/* two products accumulated in 32 bits (wrapping), then sqrshrn #15 */
static int32_t mac2(int32_t a, int32_t ka, int32_t b, int32_t kb) {
  uint32_t acc = (uint32_t)(a * ka) + (uint32_t)(b * kb);
  return sat16(((int64_t)(int32_t)acc + (1 << 14)) >> 15);
}

static q15c cadd(q15c a, q15c b) { return (q15c){sat16(a.re + b.re), sat16(a.im + b.im)}; }
static q15c csub(q15c a, q15c b) { return (q15c){sat16(a.re - b.re), sat16(a.im - b.im)}; }
/* ~ i z and ~ -i z */
static q15c mul_pi(q15c z) { return (q15c){rdm(z.im, -32768), rdm(z.re, 32767)}; }
static q15c mul_mi(q15c z) { return (q15c){rdm(z.im, 32767), rdm(z.re, -32768)}; }

enum { C8 = 23170, C16 = 30273, S16 = 12539 };

/* ~ c (1 - i) z and ~ -c (1 + i) z, c = cos(pi/4): a real-constant product
 * whose imaginary part is itself a rotated sqrdmulh, folded into one
 * 32-bit accumulate */
static q15c mul_w8(q15c z) {
  return (q15c){mac2(z.re, C8, rdm(z.im, C8), 32767), mac2(z.im, C8, rdm(z.re, C8), -32768)};
}
static q15c mul_w8_3(q15c z) {
  return (q15c){mac2(z.re, -C8, rdm(z.im, -C8), -32768), mac2(z.im, -C8, rdm(z.re, -C8), 32767)};
}
/* (wr + i wi) z with one rounding per component */
static q15c mul_w(q15c z, int32_t wr, int32_t wi) {
  return (q15c){mac2(z.re, wr, z.im, -wi), mac2(z.im, wr, z.re, wi)};
}

/* ---- codelets: x[0..r) already pre-scaled; forward order ---- */
static void dft2(const q15c *a, q15c *y) {
  y[0] = cadd(a[0], a[1]);
  y[1] = csub(a[0], a[1]);
}

static void dft4(const q15c *a, q15c *y) {
  const q15c s02 = cadd(a[0], a[2]), s13 = cadd(a[1], a[3]);
  const q15c d02 = csub(a[0], a[2]), j13 = mul_pi(csub(a[1], a[3]));
  y[0] = cadd(s02, s13);
  y[2] = csub(s02, s13);
  y[1] = csub(d02, j13);
  y[3] = cadd(d02, j13);
}

static void dft8(const q15c *a, q15c *y) {
  q15c p[4], m[4];
  for (int k = 0; k < 4; ++k) {
    p[k] = cadd(a[k], a[k + 4]);
    m[k] = csub(a[k], a[k + 4]);
  }
  const q15c e0 = cadd(p[0], p[2]), e1 = cadd(p[1], p[3]);
  y[0] = cadd(e0, e1);
  y[4] = csub(e0, e1);
  const q15c d = csub(p[0], p[2]), jd = mul_pi(csub(p[1], p[3]));
  y[2] = csub(d, jd);
  y[6] = cadd(d, jd);
  const q15c z = cadd(m[1], m[3]), w = csub(m[1], m[3]);
  const q15c rd = {rdm(w.re, C8), rdm(w.im, C8)};
  /* ~ i (M2 + c Z) and ~ i (M2 - c Z) */
  const q15c x = {mac2(m[2].im, -32768, z.im, -C8), mac2(m[2].re, 32767, z.re, C8)};
  const q15c x2 = {mac2(m[2].im, -32768, z.im, C8), mac2(m[2].re, 32767, z.re, -C8)};
  const q15c u = cadd(m[0], rd), v = csub(m[0], rd);
  y[1] = csub(u, x);
  y[7] = cadd(u, x);
  y[3] = cadd(v, x2);
  y[5] = csub(v, x2);
}

/* fixed-point split-radix 16 */
static void dft16(const q15c *a, q15c *y) {
  q15c p[8], m[8];
  for (int k = 0; k < 8; ++k) {
    p[k] = cadd(a[k], a[k + 8]);
    m[k] = csub(a[k], a[k + 8]);
  }
  /* even outputs: length-8 split of p */
  const q15c s04 = cadd(p[0], p[4]), s26 = cadd(p[2], p[6]);
  const q15c s15 = cadd(p[1], p[5]), s37 = cadd(p[3], p[7]);
  const q15c e0 = cadd(s04, s26), e1 = cadd(s15, s37);
  y[0] = cadd(e0, e1);
  y[8] = csub(e0, e1);
  const q15c A = csub(s04, s26), jB = mul_pi(csub(s15, s37));
  y[4] = csub(A, jB);
  y[12] = cadd(A, jB);
  const q15c C = csub(p[0], p[4]), jD = mul_pi(csub(p[2], p[6]));
  const q15c kE = mul_w8(csub(p[1], p[5])), kF = mul_w8_3(csub(p[3], p[7]));
  const q15c g1 = csub(C, jD), g2 = cadd(C, jD);
  const q15c h = cadd(kE, kF), h2 = mul_mi(csub(kF, kE));
  y[2] = cadd(g1, h);
  y[10] = csub(g1, h);
  y[6] = csub(g2, h2);
  y[14] = cadd(g2, h2);
  /* odd outputs */
  const q15c j4 = mul_pi(m[4]);
  const q15c q = csub(m[0], j4), q2 = cadd(m[0], j4);
  const q15c k2 = mul_w8(m[2]), k6 = mul_w8_3(m[6]);
  const q15c r = cadd(k2, k6), r2 = mul_mi(csub(k6, k2));
  const q15c j5 = mul_pi(m[5]), j7 = mul_pi(m[7]);
  const q15c u = csub(m[1], j5), u2 = cadd(m[1], j5);
  const q15c v = csub(m[3], j7), v2 = cadd(m[3], j7);
  const q15c l1 = mul_w(u, C16, -S16), l3 = mul_w(v, S16, -C16);
  const q15c l3b = mul_w(u2, S16, -C16), l9 = mul_w(v2, -C16, S16);
  const q15c qr = cadd(q, r), qmr = csub(q, r);
  const q15c ls = cadd(l1, l3), ld = mul_mi(csub(l3, l1));
  y[1] = cadd(qr, ls);
  y[9] = csub(qr, ls);
  y[5] = csub(qmr, ld);
  y[13] = cadd(qmr, ld);
  const q15c qa = csub(q2, r2), qb = cadd(q2, r2);
  const q15c ls2 = cadd(l3b, l9), ld2 = mul_mi(csub(l9, l3b));
  y[3] = cadd(qa, ls2);
  y[11] = csub(qa, ls2);
  y[7] = csub(qb, ld2);
  y[15] = cadd(qb, ld2);
}

static int ilog2(int r) {
  int s = 0;
  while ((1 << s) < r) ++s;
  return s;
}

/* one codelet of length r on pre-scaled inputs; the backward codelet
 * returns the forward one's outputs in reversed index order */
static void codelet(int r, int dir, const q15c *a, q15c *out) {
  q15c y[16];
  switch (r) {
    case 1: y[0] = a[0]; break;
    case 2: dft2(a, y); break;
    case 4: dft4(a, y); break;
    case 8: dft8(a, y); break;
    default: dft16(a, y); break;
  }
  for (int k = 0; k < r; ++k) out[k] = y[dir < 0 ? k : (r - k) % r];
}

static q15c load(const int16_t *p, int64_t k, int s) {
  return (q15c){rshr(p[2 * k], s), rshr(p[2 * k + 1], s)};
}
static void store(int16_t *p, int64_t k, q15c v) {
  p[2 * k] = (int16_t)v.re;
  p[2 * k + 1] = (int16_t)v.im;
}

static int16_t cvt_q15(double x) {
  const float f = (float)x * 32768.0f;
  const double t = trunc((double)f);
  return (int16_t)(t > 32767.0 ? 32767 : (t < -32768.0 ? -32768 : (int32_t)t));
}

/* stage-2 twiddle table: for j = 1..m-1, i = 1..15: (c, s, cvt(-s), c) */
void oracle_q15_twiddles(int64_t n, int dir, int16_t *w) {
  const int64_t m = n / 16;
  const double base = (double)dir * 2.0 * M_PI / (double)n;
  int64_t x = 0;
  for (int64_t j = 1; j < m; ++j)
    for (int64_t i = 1; i < 16; ++i) {
      const double ang = base * (double)i * (double)j;
      const double a = cos(ang), b = sin(ang);
      w[x++] = cvt_q15(a);
      w[x++] = cvt_q15(b);
      w[x++] = cvt_q15(-b);
      w[x++] = cvt_q15(a);
    }
}

/* Q0.15 C2C of power-of-two n in [1, 256]; returns 0, or -1 if n is not
 * supported */
int oracle_q15_c2c(const int16_t *in, int16_t *out, int64_t n, int64_t howmany, int64_t idist,
                   int64_t odist, int dir) {
  if (n < 1 || n > 256 || (n & (n - 1))) return -1;
  if (n <= 16) {
    const int s = ilog2((int)n);
    for (int64_t b = 0; b < howmany; ++b) {
      q15c a[16], y[16];
      for (int k = 0; k < n; ++k) a[k] = load(in + 2 * b * idist, k, s);
      codelet((int)n, dir, a, y);
      for (int k = 0; k < n; ++k) store(out + 2 * b * odist, k, y[k]);
    }
    return 0;
  }
  const int m = (int)(n / 16), sm = ilog2(m);
  int16_t *w = (int16_t *)malloc(sizeof(int16_t) * 4 * 15 * (size_t)(m - 1));
  oracle_q15_twiddles(n, dir, w);
  for (int64_t b = 0; b < howmany; ++b) {
    const int16_t *x = in + 2 * b * idist;
    int16_t *yb = out + 2 * b * odist;
    q15c tmp[256];
    for (int c = 0; c < 16; ++c) { /* stage 1: length-m codelets down the columns */
      q15c a[16], y[16];
      for (int q = 0; q < m; ++q) a[q] = load(x, c + 16 * q, sm);
      codelet(m, dir, a, y);
      for (int k = 0; k < m; ++k) tmp[c + 16 * k] = y[k];
    }
    for (int j = 0; j < m; ++j) { /* stage 2: twiddled 16-point rows */
      q15c a[16], y[16];
      for (int i = 0; i < 16; ++i) {
        const q15c v = {rshr(tmp[16 * j + i].re, 4), rshr(tmp[16 * j + i].im, 4)};
        if (j == 0 || i == 0) {
          a[i] = v;
        } else {
          const int16_t *t = w + 4 * (15 * (j - 1) + (i - 1));
          a[i] = (q15c){mac2(v.re, t[0], v.im, t[2]), mac2(v.re, t[1], v.im, t[3])};
        }
      }
      codelet(16, dir, a, y);
      for (int k = 0; k < 16; ++k) store(yb, j + (int64_t)m * k, y[k]);
    }
  }
  free(w);
  return 0;
}
