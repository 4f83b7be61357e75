/*
 * Bit-exact CPU restatement of the reference's fixed-point C2C, R2C and
 * C2R paths, Q0.15 and Q0.7 -- TEST INFRASTRUCTURE ONLY (same rules as oracle.c: only tests/
 * and the CPU-baseline leg of bench.py load it, to check results).
 *
 * What is restated (arm/perf-libs-fft), for lanes of B = 16 or 8 bits:
 *   Arithmetic semantics (src/providers/jit/print_algo.cpp:1228-1230,
 *   src/providers/jit/emit.hpp:150-175 and :370-425, constant lowering
 *   print_algo.cpp:2150-2290):
 *     - every codelet input is pre-scaled by a rounding shift right by
 *       log2(radix) (srshr), so a whole transform is scaled by 1/N;
 *     - additions and subtractions saturate to B bits (sqadd / sqsub);
 *     - a multiply by a real constant k (a Q0.(B-1) value) is
 *       (a k + 2^(B-2)) >> (B-1), saturated: sqrdmulh for Q0.15, smull +
 *       sqrshrn #7 for Q0.7 (the two agree on this formula); multiplying by
 *       +-i swaps re/im and uses k = -2^(B-1) or 2^(B-1) - 1 on the lanes;
 *     - a complex product with a twiddle (and the fused constant products
 *       of the radix-8/16 codelets) is two B x B products accumulated in a
 *       2B-bit lane (smull / smlal / smlsl, wrapping at 2B bits) and
 *       narrowed once by a rounding, saturating shift by B - 1 (sqrshrn).
 *   Codelets: radix 2, 4, 8 and the fixed-point split-radix 16
 *   (src/providers/jit/split_radix_z16.cpp, selected for fixed point by
 *   src/providers/jit/wfta_nfact.cpp:89-97); the backward codelet of
 *   length r produces, at output k, the forward codelet's output r-k.
 *   Composition: the reference's ESTIMATE plan (planner/planner.cpp:51-175,
 *   first applicable strategy; base kernels {2, 4, 8, 16},
 *   providers/aot/aot_kernel_data.cpp:296-300):
 *     N <= 16        one codelet per member;
 *     N = 16 m       (m <= 16) cooley_tukey_ab(16): length-m codelets down
 *                    the 16 columns x[c + 16 q], then per row j a 16-point
 *                    codelet whose inputs i >= 1 are multiplied by the
 *                    twiddle W_N^{dir i j} (row 0 untwiddled), writing
 *                    y[j + m k] (planner/strategies/cooley_tukey.hpp:82-143,
 *                    622-680);
 *     N = 256 m'     (m' = 2..16) cooley_tukey_ab(16) whose length-16 m'
 *                    sub-transforms are cooley_tukey_ac(16)
 *                    (cooley_tukey.hpp:331-385, 682-748): length-m' codelets
 *                    down the 256 columns x[c + 256 q] into b1[c + 256 k];
 *                    then for column t < 16 and row i0 < m' a 16-point
 *                    codelet over b1[256 i0 + t + 16 i], inputs i >= 1 of
 *                    rows i0 >= 1 twiddled by W_{16 m'}^{dir i i0}, into
 *                    b0[16 i0 + t + 16 m' k]; then the twiddled 16-point
 *                    rows of the N = 16 m case over b0.
 *   Twiddles: cvt(x) = sat(trunc(float(x) * 2^(B-1))) of cos and sin of the
 *   angle (src/generate_twiddles.hpp:72-132, src/plfft_convert.hpp:36-54),
 *   stored as the premultiplied pairs (c, s), (-s, c).
 *
 * Parity pin: tests/golden/q15_reference.npz and q7_reference.npz hold
 * outputs of the reference's own NEON kernels composed as its ESTIMATE
 * plans (executed from their source text by tests/golden/neon_a64.py);
 * tests/test_q15.py and tests/test_q7.py require this file to match them
 * bit for bit; q15_r2c_reference.npz and q7_r2c_reference.npz pin the R2C
 * (fixed_r2c below) the same way (tests/test_fixed_r2c.py), and
 * q15_c2r_reference.npz and q7_c2r_reference.npz the C2R (fixed_c2r,
 * tests/test_fixed_c2r.py).
 *
 * Data: interleaved (re, im) of int16 (Q0.15) or int8 (Q0.7), members
 * idist/odist complex elements apart, unit element stride (R2C: real
 * inputs and complex outputs with their own strides).  Members are
 * independent: the batch loops run OpenMP-parallel.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int32_t re, im;
} fc;

/* lane format */
typedef struct {
  int bits;          /* 16 or 8 */
  int32_t lo, hi;    /* saturation bounds */
  int32_t one, mone; /* the constants 1 - 2^-(B-1) and -1 */
  int32_t c8, c16, s16;
} fmt;

static fmt make_fmt(int bits);

static int32_t sat(const fmt *f, int64_t v) { return v > f->hi ? f->hi : (v < f->lo ? f->lo : (int32_t)v); }
static int32_t rshr(int32_t v, int s) { return (v + (1 << (s - 1))) >> s; }
/* multiply by a real constant, one rounding */
static int32_t rdm(const fmt *f, int32_t a, int32_t k) {
  return sat(f, ((int64_t)a * k + ((int64_t)1 << (f->bits - 2))) >> (f->bits - 1));
}
/* two products accumulated in a 2B-bit lane (wrapping), one rounding narrow */
static int32_t mac2(const fmt *f, int32_t a, int32_t ka, int32_t b, int32_t kb) {
  const int w = 2 * f->bits;
  int64_t acc = (int64_t)a * ka + (int64_t)b * kb;
  const int64_t m = (int64_t)1 << w;
  acc = ((acc % m) + m) % m;
  if (acc >= m / 2) acc -= m;
  return sat(f, (acc + ((int64_t)1 << (f->bits - 2))) >> (f->bits - 1));
}

static fc cadd(const fmt *f, fc a, fc b) { return (fc){sat(f, a.re + b.re), sat(f, a.im + b.im)}; }
static fc csub(const fmt *f, fc a, fc b) { return (fc){sat(f, a.re - b.re), sat(f, a.im - b.im)}; }
/* ~ i z and ~ -i z */
static fc mul_pi(const fmt *f, fc z) { return (fc){rdm(f, z.im, f->mone), rdm(f, z.re, f->one)}; }
static fc mul_mi(const fmt *f, fc z) { return (fc){rdm(f, z.im, f->one), rdm(f, z.re, f->mone)}; }

/* ~ c (1 - i) z and ~ -c (1 + i) z, c = cos(pi/4): a real-constant product
 * whose imaginary part is itself a rotated constant product, folded into one
 * accumulate */
static fc mul_w8(const fmt *f, fc z) {
  return (fc){mac2(f, z.re, f->c8, rdm(f, z.im, f->c8), f->one),
              mac2(f, z.im, f->c8, rdm(f, z.re, f->c8), f->mone)};
}
static fc mul_w8_3(const fmt *f, fc z) {
  return (fc){mac2(f, z.re, -f->c8, rdm(f, z.im, -f->c8), f->mone),
              mac2(f, z.im, -f->c8, rdm(f, z.re, -f->c8), f->one)};
}
/* (wr + i wi) z with one rounding per component */
static fc mul_w(const fmt *f, fc z, int32_t wr, int32_t wi) {
  return (fc){mac2(f, z.re, wr, z.im, -wi), mac2(f, z.im, wr, z.re, wi)};
}

/* ---- codelets: x[0..r) already pre-scaled; forward order ---- */
static void dft2(const fmt *f, const fc *a, fc *y) {
  y[0] = cadd(f, a[0], a[1]);
  y[1] = csub(f, a[0], a[1]);
}

static void dft4(const fmt *f, const fc *a, fc *y) {
  const fc s02 = cadd(f, a[0], a[2]), s13 = cadd(f, a[1], a[3]);
  const fc d02 = csub(f, a[0], a[2]), j13 = mul_pi(f, csub(f, a[1], a[3]));
  y[0] = cadd(f, s02, s13);
  y[2] = csub(f, s02, s13);
  y[1] = csub(f, d02, j13);
  y[3] = cadd(f, d02, j13);
}

static void dft8(const fmt *f, const fc *a, fc *y) {
  fc p[4], m[4];
  for (int k = 0; k < 4; ++k) {
    p[k] = cadd(f, a[k], a[k + 4]);
    m[k] = csub(f, a[k], a[k + 4]);
  }
  const fc e0 = cadd(f, p[0], p[2]), e1 = cadd(f, p[1], p[3]);
  y[0] = cadd(f, e0, e1);
  y[4] = csub(f, e0, e1);
  const fc d = csub(f, p[0], p[2]), jd = mul_pi(f, csub(f, p[1], p[3]));
  y[2] = csub(f, d, jd);
  y[6] = cadd(f, d, jd);
  const fc z = cadd(f, m[1], m[3]), w = csub(f, m[1], m[3]);
  const fc rd = {rdm(f, w.re, f->c8), rdm(f, w.im, f->c8)};
  /* ~ i (M2 + c Z) and ~ i (M2 - c Z) */
  const fc x = {mac2(f, m[2].im, f->mone, z.im, -f->c8), mac2(f, m[2].re, f->one, z.re, f->c8)};
  const fc x2 = {mac2(f, m[2].im, f->mone, z.im, f->c8), mac2(f, m[2].re, f->one, z.re, -f->c8)};
  const fc u = cadd(f, m[0], rd), v = csub(f, m[0], rd);
  y[1] = csub(f, u, x);
  y[7] = cadd(f, u, x);
  y[3] = cadd(f, v, x2);
  y[5] = csub(f, v, x2);
}

/* fixed-point split-radix 16 */
static void dft16(const fmt *f, const fc *a, fc *y) {
  fc p[8], m[8];
  for (int k = 0; k < 8; ++k) {
    p[k] = cadd(f, a[k], a[k + 8]);
    m[k] = csub(f, a[k], a[k + 8]);
  }
  /* even outputs: length-8 split of p */
  const fc s04 = cadd(f, p[0], p[4]), s26 = cadd(f, p[2], p[6]);
  const fc s15 = cadd(f, p[1], p[5]), s37 = cadd(f, p[3], p[7]);
  const fc e0 = cadd(f, s04, s26), e1 = cadd(f, s15, s37);
  y[0] = cadd(f, e0, e1);
  y[8] = csub(f, e0, e1);
  const fc A = csub(f, s04, s26), jB = mul_pi(f, csub(f, s15, s37));
  y[4] = csub(f, A, jB);
  y[12] = cadd(f, A, jB);
  const fc C = csub(f, p[0], p[4]), jD = mul_pi(f, csub(f, p[2], p[6]));
  const fc kE = mul_w8(f, csub(f, p[1], p[5])), kF = mul_w8_3(f, csub(f, p[3], p[7]));
  const fc g1 = csub(f, C, jD), g2 = cadd(f, C, jD);
  const fc h = cadd(f, kE, kF), h2 = mul_mi(f, csub(f, kF, kE));
  y[2] = cadd(f, g1, h);
  y[10] = csub(f, g1, h);
  y[6] = csub(f, g2, h2);
  y[14] = cadd(f, g2, h2);
  /* odd outputs */
  const fc j4 = mul_pi(f, m[4]);
  const fc q = csub(f, m[0], j4), q2 = cadd(f, m[0], j4);
  const fc k2 = mul_w8(f, m[2]), k6 = mul_w8_3(f, m[6]);
  const fc r = cadd(f, k2, k6), r2 = mul_mi(f, csub(f, k6, k2));
  const fc j5 = mul_pi(f, m[5]), j7 = mul_pi(f, m[7]);
  const fc u = csub(f, m[1], j5), u2 = cadd(f, m[1], j5);
  const fc v = csub(f, m[3], j7), v2 = cadd(f, m[3], j7);
  const fc l1 = mul_w(f, u, f->c16, -f->s16), l3 = mul_w(f, v, f->s16, -f->c16);
  const fc l3b = mul_w(f, u2, f->s16, -f->c16), l9 = mul_w(f, v2, -f->c16, f->s16);
  const fc qr = cadd(f, q, r), qmr = csub(f, q, r);
  const fc ls = cadd(f, l1, l3), ld = mul_mi(f, csub(f, l3, l1));
  y[1] = cadd(f, qr, ls);
  y[9] = csub(f, qr, ls);
  y[5] = csub(f, qmr, ld);
  y[13] = cadd(f, qmr, ld);
  const fc qa = csub(f, q2, r2), qb = cadd(f, q2, r2);
  const fc ls2 = cadd(f, l3b, l9), ld2 = mul_mi(f, csub(f, l9, l3b));
  y[3] = cadd(f, qa, ls2);
  y[11] = csub(f, qa, ls2);
  y[7] = csub(f, qb, ld2);
  y[15] = cadd(f, qb, ld2);
}

static int ilog2(int r) {
  int s = 0;
  while ((1 << s) < r) ++s;
  return s;
}

/* one codelet of length r on pre-scaled inputs; the backward codelet
 * returns the forward one's outputs in reversed index order */
static void codelet(const fmt *f, int r, int dir, const fc *a, fc *out) {
  fc y[16];
  switch (r) {
    case 1: y[0] = a[0]; break;
    case 2: dft2(f, a, y); break;
    case 4: dft4(f, a, y); break;
    case 8: dft8(f, a, y); break;
    default: dft16(f, a, y); break;
  }
  for (int k = 0; k < r; ++k) out[k] = y[dir < 0 ? k : (r - k) % r];
}

static int32_t cvt(const fmt *f, double x) {
  const float v = (float)x * (float)(1 << (f->bits - 1));
  return sat(f, (int64_t)trunc((double)v));
}

static fmt make_fmt(int bits) {
  fmt f;
  f.bits = bits;
  f.hi = (1 << (bits - 1)) - 1;
  f.lo = -(1 << (bits - 1));
  f.one = f.hi;
  f.mone = f.lo;
  f.c8 = cvt(&f, cos(M_PI / 4));
  f.c16 = cvt(&f, cos(M_PI / 8));
  f.s16 = cvt(&f, sin(M_PI / 8));
  return f;
}

/* premultiplied twiddle table of a radix-16 level over n1 rows, angle
 * dir 2 pi i j / (16 n1): for j = 1..n1-1, i = 1..15: (c, s, cvt(-s), c) */
static void twiddles16(const fmt *f, int64_t n1, int dir, int32_t *w) {
  const double base = (double)dir * 2.0 * M_PI / (double)(16 * n1);
  int64_t x = 0;
  for (int64_t j = 1; j < n1; ++j)
    for (int64_t i = 1; i < 16; ++i) {
      const double ang = base * (double)i * (double)j;
      const double a = cos(ang), b = sin(ang);
      w[x++] = cvt(f, a);
      w[x++] = cvt(f, b);
      w[x++] = cvt(f, -b);
      w[x++] = cvt(f, a);
    }
}

/* a 16-point codelet on pre-scaled inputs, the inputs i >= 1 multiplied by
 * row `row` of a premultiplied table (row 0: untwiddled) */
static void twiddled16(const fmt *f, int dir, const fc *v, int64_t row, const int32_t *w, fc *out) {
  fc a[16];
  for (int i = 0; i < 16; ++i) {
    const fc s = {rshr(v[i].re, 4), rshr(v[i].im, 4)};
    if (row == 0 || i == 0) {
      a[i] = s;
    } else {
      const int32_t *t = w + 4 * (15 * (row - 1) + (i - 1));
      a[i] = (fc){mac2(f, s.re, t[0], s.im, t[2]), mac2(f, s.re, t[1], s.im, t[3])};
    }
  }
  codelet(f, 16, dir, a, out);
}

typedef struct {
  const fmt *f;
  int bits;
  const void *in;
  void *out;
} io;

static fc ld(int bits, const void *p, int64_t k) {
  if (bits == 16) {
    const int16_t *q = (const int16_t *)p;
    return (fc){q[2 * k], q[2 * k + 1]};
  }
  const int8_t *q = (const int8_t *)p;
  return (fc){q[2 * k], q[2 * k + 1]};
}
static void st(int bits, void *p, int64_t k, fc v) {
  if (bits == 16) {
    int16_t *q = (int16_t *)p;
    q[2 * k] = (int16_t)v.re;
    q[2 * k + 1] = (int16_t)v.im;
  } else {
    int8_t *q = (int8_t *)p;
    q[2 * k] = (int8_t)v.re;
    q[2 * k + 1] = (int8_t)v.im;
  }
}

/* fixed-point C2C of power-of-two n in [1, 4096]; returns 0, or -1 if n is
 * not supported */
static int fixed_c2c(int bits, const void *in, void *out, int64_t n, int64_t howmany, int64_t idist,
                     int64_t odist, int dir) {
  if (n < 1 || n > 4096 || (n & (n - 1))) return -1;
  const fmt F = make_fmt(bits), *f = &F;
  const size_t esz = (size_t)(bits / 4); /* bytes per complex element */
  if (n <= 16) {
    const int s = ilog2((int)n);
#pragma omp parallel for schedule(static)
    for (int64_t b = 0; b < howmany; ++b) {
      fc a[16], y[16];
      const void *x = (const char *)in + esz * (size_t)(b * idist);
      for (int k = 0; k < n; ++k) {
        const fc v = ld(bits, x, k);
        a[k] = s ? (fc){rshr(v.re, s), rshr(v.im, s)} : v;
      }
      codelet(f, (int)n, dir, a, y);
      for (int k = 0; k < n; ++k) st(bits, (char *)out + esz * (size_t)(b * odist), k, y[k]);
    }
    return 0;
  }
  const int64_t m = n / 16;                        /* rows of the outer radix-16 level */
  const int64_t m2 = n > 256 ? n / 256 : 0;        /* rows of the inner radix-16 level */
  const int64_t first = n > 256 ? m2 : m;          /* length of the first-stage codelets */
  const int64_t cols = n / first;                  /* number of first-stage columns */
  const int sf = ilog2((int)first);
  int32_t *w = (int32_t *)malloc(sizeof(int32_t) * 4 * 15 * (size_t)(m > 1 ? m - 1 : 1));
  int32_t *w2 = (int32_t *)malloc(sizeof(int32_t) * 4 * 15 * (size_t)(m2 > 1 ? m2 - 1 : 1));
  twiddles16(f, m, dir, w);
  if (m2) twiddles16(f, m2, dir, w2);
#pragma omp parallel
  {
  fc *b1 = (fc *)malloc(sizeof(fc) * (size_t)n); /* per-thread scratch */
  fc *b0 = (fc *)malloc(sizeof(fc) * (size_t)n);
#pragma omp for schedule(static)
  for (int64_t b = 0; b < howmany; ++b) {
    const void *x = (const char *)in + esz * (size_t)(b * idist);
    void *yb = (char *)out + esz * (size_t)(b * odist);
    /* first stage: length-`first` codelets down the columns x[c + cols q] */
    for (int64_t c = 0; c < cols; ++c) {
      fc a[16], y[16];
      for (int q = 0; q < first; ++q) {
        const fc v = ld(bits, x, c + cols * q);
        a[q] = (fc){rshr(v.re, sf), rshr(v.im, sf)};
      }
      codelet(f, (int)first, dir, a, y);
      for (int k = 0; k < first; ++k) b1[c + cols * k] = y[k];
    }
    const fc *rows = b1;
    if (m2) { /* inner radix-16 level: column t, row i0 */
      for (int64_t i0 = 0; i0 < m2; ++i0)
        for (int t = 0; t < 16; ++t) {
          fc v[16], y[16];
          for (int i = 0; i < 16; ++i) v[i] = b1[256 * i0 + t + 16 * i];
          twiddled16(f, dir, v, i0, w2, y);
          for (int k = 0; k < 16; ++k) b0[16 * i0 + t + 16 * m2 * k] = y[k];
        }
      rows = b0;
    }
    for (int64_t j = 0; j < m; ++j) { /* outer radix-16 level: twiddled rows */
      fc y[16];
      twiddled16(f, dir, rows + 16 * j, j, w, y);
      for (int k = 0; k < 16; ++k) st(bits, yb, j + m * k, y[k]);
    }
  }
  free(b1);
  free(b0);
  }
  free(w);
  free(w2);
  return 0;
}

/* The reference's 8-point real-input codelet (plfft_8_*_hjjnfoh, forward):
 * with a_k = x_k pre-shifted by 3, d/s = saturating differences / sums,
 *   g = d15 - d37, h = d15 + d37, e1 = s15 - s37, f1 = s15 + s37,
 *   p = s04 - s26, q = s04 + s26,
 *   X0 = (q + f1, 0), X4 = (q - f1, 0), X2 = (rdm(p, 1), rdm(e1, -1)),
 *   X1 = (rdm(d04 + rdm(g, c8), 1), rdm(d26 + rdm(h, c8), -1)),
 *   X3 = (d04 - rdm(g, c8), d26 - rdm(h, c8)),
 * where 1 and -1 are the format's 1 - 2^-(B-1) and -1 (the uun, us and gs
 * variants).  Bins 1 and 3 round differently from the complex codelet on
 * (x, 0); bins 5..7 are not used. */
static void real8(const fmt *f, const int32_t *x, fc *y) {
  int32_t a[8];
  for (int k = 0; k < 8; ++k) a[k] = rshr(x[k], 3);
  const int32_t d15 = sat(f, a[1] - a[5]), s15 = sat(f, a[1] + a[5]);
  const int32_t d26 = sat(f, a[2] - a[6]), s26 = sat(f, a[2] + a[6]);
  const int32_t d37 = sat(f, a[3] - a[7]), s37 = sat(f, a[3] + a[7]);
  const int32_t d04 = sat(f, a[0] - a[4]), s04 = sat(f, a[0] + a[4]);
  const int32_t e1 = sat(f, s15 - s37), f1 = sat(f, s15 + s37);
  const int32_t g = sat(f, d15 - d37), h = sat(f, d15 + d37);
  const int32_t rg = rdm(f, g, f->c8), rh = rdm(f, h, f->c8);
  const int32_t p = sat(f, s04 - s26), q = sat(f, s04 + s26);
  y[0] = (fc){sat(f, q + f1), 0};
  y[4] = (fc){sat(f, q - f1), 0};
  y[2] = (fc){rdm(f, p, f->one), rdm(f, e1, f->mone)};
  y[1] = (fc){rdm(f, sat(f, d04 + rg), f->one), rdm(f, sat(f, d26 + rh), f->mone)};
  y[3] = (fc){sat(f, d04 - rg), sat(f, d26 - rh)};
  for (int k = 5; k < 8; ++k) y[k] = (fc){0, 0};
}

/* The reference's 8-point real-input codelet in its unit-output-distance
 * batch variant (plfft_8_*_hjjnfoh_uu / _gu, which also runs as the first
 * stage of every larger R2C plan, vectorised across its columns): the same
 * sums as real8, with
 *   X2 = (p, -rdm(e1, 1)), X1 = (d04 + rdm(g, c8), -rdm(d26 + rdm(h, c8), 1)),
 *   X3 = (d04 - rdm(g, c8), rdm(d26 - rdm(h, c8), 1))
 * (negations saturating). */
static void real8_uo(const fmt *f, const int32_t *x, fc *y) {
  int32_t a[8];
  for (int k = 0; k < 8; ++k) a[k] = rshr(x[k], 3);
  const int32_t d15 = sat(f, a[1] - a[5]), s15 = sat(f, a[1] + a[5]);
  const int32_t d26 = sat(f, a[2] - a[6]), s26 = sat(f, a[2] + a[6]);
  const int32_t d37 = sat(f, a[3] - a[7]), s37 = sat(f, a[3] + a[7]);
  const int32_t d04 = sat(f, a[0] - a[4]), s04 = sat(f, a[0] + a[4]);
  const int32_t e1 = sat(f, s15 - s37), f1 = sat(f, s15 + s37);
  const int32_t g = sat(f, d15 - d37), h = sat(f, d15 + d37);
  const int32_t rg = rdm(f, g, f->c8), rh = rdm(f, h, f->c8);
  const int32_t p = sat(f, s04 - s26), q = sat(f, s04 + s26);
  y[0] = (fc){sat(f, q + f1), 0};
  y[4] = (fc){sat(f, q - f1), 0};
  y[2] = (fc){p, sat(f, -(int64_t)rdm(f, e1, f->one))};
  y[1] = (fc){sat(f, d04 + rg), sat(f, -(int64_t)rdm(f, sat(f, d26 + rh), f->one))};
  y[3] = (fc){sat(f, d04 - rg), rdm(f, sat(f, d26 - rh), f->one)};
  for (int k = 5; k < 8; ++k) y[k] = (fc){0, 0};
}

/* The 4-point real-input codelet of the single-member and strided-output
 * variants (plfft_4_*_hjjnfoh / rppnfoh, uun, us, gs): X0, X2 as the complex
 * codelet, X1 = (rdm(a0 - a2, 1), rdm(a1 - a3, -1)).  The unit-output-distance
 * variants (uu, gu) compute X1 as the complex codelet does. */
static void real4(const fmt *f, const int32_t *x, fc *y) {
  int32_t a[4];
  for (int k = 0; k < 4; ++k) a[k] = rshr(x[k], 2);
  const int32_t s02 = sat(f, a[0] + a[2]), d02 = sat(f, a[0] - a[2]);
  const int32_t s13 = sat(f, a[1] + a[3]), d13 = sat(f, a[1] - a[3]);
  y[0] = (fc){sat(f, s02 + s13), 0};
  y[2] = (fc){sat(f, s02 - s13), 0};
  y[1] = (fc){rdm(f, d02, f->one), rdm(f, d13, f->mone)};
  y[3] = (fc){0, 0};
}

/* real-input codelet of length r <= 16 on x.  uo selects the
 * unit-output-distance kernel variant (uu, gu: a batch whose members are
 * adjacent in the output), which is also the first stage of the larger
 * plans; the others (uun, us, gs) use real8 and real4.  Lengths 2 and 16, and
 * length 4 of the uo variants, are the complex codelet on (x, 0). */
static void real_codelet(const fmt *f, int r, int uo, const int32_t *x, fc *y) {
  if (r == 8) {
    if (uo)
      real8_uo(f, x, y);
    else
      real8(f, x, y);
    return;
  }
  if (r == 4 && !uo) {
    real4(f, x, y);
    return;
  }
  const int s = ilog2(r);
  fc a[16];
  for (int k = 0; k < r; ++k) a[k] = (fc){rshr(x[k], s), 0};
  codelet(f, r, -1, a, y);
}

/* fixed-point R2C (forward) of power-of-two n in [2, 4096]: the reference's
 * R2C plans run the same levels as the C2C ones on the real input (imaginary
 * parts zero), but each twiddled radix-16 level computes only the rows
 * r <= rows/2 of its sub-spectra and writes row rows - r (r >= 1) as the
 * conjugate of row r with the codelet outputs reversed: output k of row
 * rows - r is conj(output 15 - k of row r), from X[L - b] = conj(X[b]) for
 * the length-L sub-spectrum of a real sequence (the R2C twiddled levels
 * with conjugate-reversed second output,
 * planner/strategies/cooley_tukey.hpp:145-248, 386-470, and the kernels
 * plfft_ab / ac _q15_jjjtfj_dit).  The length-n/16 and n/256 first-stage
 * codelets read only bins <= half their length: the reference's real-input
 * kernels in their uu variant (real_codelet with uo set).  A plan of n <= 16
 * is one real-input kernel whose variant follows the batch layout
 * (providers/aot/aot_kernel_data.cpp:188-252): uu or gu when the batch has
 * more than one member and odist is 1, else uun, us or gs.  Outputs: bins
 * 0..n/2, ostride complex elements apart, members odist apart; inputs
 * istride reals apart, members idist apart. */
static int fixed_r2c(int bits, const void *in, void *out, int64_t n, int64_t howmany, int64_t istride,
                     int64_t idist, int64_t ostride, int64_t odist) {
  if (n < 2 || n > 4096 || (n & (n - 1))) return -1;
  const fmt F = make_fmt(bits), *f = &F;
  const size_t esz = (size_t)(bits / 4), rsz = (size_t)(bits / 8);
  const int64_t h = n / 2 + 1;
  int32_t *w = NULL, *w2 = NULL;
  const int64_t m = n / 16, m2 = n > 256 ? n / 256 : 0, first = n > 256 ? m2 : m, cols = n > 16 ? n / first : 0;
  if (n > 16) {
    w = (int32_t *)malloc(sizeof(int32_t) * 4 * 15 * (size_t)(m > 1 ? m - 1 : 1));
    w2 = (int32_t *)malloc(sizeof(int32_t) * 4 * 15 * (size_t)(m2 > 1 ? m2 - 1 : 1));
    twiddles16(f, m, -1, w);
    if (m2) twiddles16(f, m2, -1, w2);
  }
#pragma omp parallel
  {
  fc *x = (fc *)malloc(sizeof(fc) * (size_t)n); /* per-thread scratch */
  fc *y = (fc *)malloc(sizeof(fc) * (size_t)n);
  fc *b1 = (fc *)malloc(sizeof(fc) * (size_t)n);
  fc *b0 = (fc *)malloc(sizeof(fc) * (size_t)n);
#pragma omp for schedule(static)
  for (int64_t b = 0; b < howmany; ++b) {
    for (int64_t k = 0; k < n; ++k) {
      const char *p = (const char *)in + rsz * (size_t)(b * idist + k * istride);
      x[k] = (fc){bits == 16 ? *(const int16_t *)p : *(const int8_t *)p, 0};
    }
    if (n <= 16) {
      int32_t r[16];
      for (int k = 0; k < n; ++k) r[k] = x[k].re;
      real_codelet(f, (int)n, howmany > 1 && odist == 1, r, y);
    } else {
      for (int64_t c = 0; c < cols; ++c) {
        int32_t r[16];
        fc yy[16];
        for (int q = 0; q < first; ++q) r[q] = x[c + cols * q].re;
        real_codelet(f, (int)first, 1, r, yy);
        for (int k = 0; k < first; ++k) b1[c + cols * k] = yy[k];
      }
      const fc *rows = b1;
      if (m2) { /* inner radix-16 level: rows i0 > m2/2 mirrored */
        for (int64_t i0 = 0; i0 <= m2 / 2; ++i0)
          for (int t = 0; t < 16; ++t) {
            fc v[16], yy[16];
            for (int i = 0; i < 16; ++i) v[i] = b1[256 * i0 + t + 16 * i];
            twiddled16(f, -1, v, i0, w2, yy);
            for (int k = 0; k < 16; ++k) {
              b0[16 * i0 + t + 16 * m2 * k] = yy[k];
              if (i0 > 0 && 2 * i0 < m2)
                b0[16 * (m2 - i0) + t + 16 * m2 * (15 - k)] = (fc){yy[k].re, -yy[k].im};
            }
          }
        rows = b0;
      }
      for (int64_t j = 0; j <= m / 2; ++j) { /* outer radix-16 level: rows j > m/2 mirrored */
        fc yy[16];
        twiddled16(f, -1, rows + 16 * j, j, w, yy);
        for (int k = 0; k < 16; ++k) {
          y[j + m * k] = yy[k];
          if (j > 0 && 2 * j < m) y[(m - j) + m * (15 - k)] = (fc){yy[k].re, -yy[k].im};
        }
      }
    }
    for (int64_t k = 0; k < h; ++k) st(bits, (char *)out + esz * (size_t)(b * odist + k * ostride), 0, y[k]);
  }
  free(x);
  free(y);
  free(b1);
  free(b0);
  }
  free(w);
  free(w2);
  return 0;
}

/* ---- C2R (backward), the reference's fixed-point real-output plans ----
 *
 * The C2R plan is the C2C decomposition run backward with decimation in
 * frequency (planner/strategies/cooley_tukey.hpp:250-323, 498-580; the
 * level call sequences of src/level_ab_t_c2r.cpp:17-99 and
 * src/level_ac_t_c2r.cpp:17-100):
 *   N <= 16       one real-output codelet;
 *   N = 16 m      a radix-16 DIF level over rows j = 0..m/2 of the Hermitian
 *                 input (row j: inputs X[j + m i], i = 0..15, those past the
 *                 stored half read as conjugates, X[j + m i] = conj(X[m (16 -
 *                 i) - j]); a backward 16-point codelet; outputs k >= 1 of
 *                 rows j >= 1 times W_N^{jk}) into b[16 j + k], then per
 *                 column k a real-output codelet of length m over b[16 j + k],
 *                 j = 0..m/2, giving x[k + 16 t];
 *   N = 256 m'    the same first level, then per column k a second radix-16
 *                 DIF level over rows i = 0..m'/2 of that column's length-m
 *                 Hermitian sequence into c[256 i + 16 q + k], then per lane
 *                 l < 256 a real-output codelet of length m' over
 *                 c[256 i + l], giving x[l + 256 t].
 * Rows j = m/2 + 1..m - 1 are not needed: the column sequences are
 * Hermitian, and each codelet conjugates what it needs.
 * Rounding, read from the kernels (plfft_*_q15_jjjnbih_*,
 * plfft_ab/ac_16_q15_jjjtbil_dif_*, plfft_*_q15_jjhnb_*; the q7 ones follow
 * the same dataflow): inputs are pre-shifted by log2 of the codelet length
 * first, and a conjugated input is then (rdm(re, 1), rdm(im, -1)); the row
 * kernels are then exactly the backward complex codelet on that column and
 * the DIF twiddle the premultiplied two-product MAC; the real-output
 * codelets of lengths 2 and 4 are the real parts of the backward complex
 * codelet, and those of lengths 8 and 16 round their constant products in
 * their own places (real_out8, real_out16). */

/* the length-r column with conjugate extension: element e of the stored
 * half is X[e * xs] (e <= r/2, or e <= h for the row form below) */
static fc cx_in(const fmt *f, fc v, int s, int conj) {
  const fc a = {s ? rshr(v.re, s) : v.re, s ? rshr(v.im, s) : v.im};
  return conj ? (fc){rdm(f, a.re, f->one), rdm(f, a.im, f->mone)} : a;
}

/* real-output codelet of length 8 on the extended, pre-shifted inputs A */
static void real_out8(const fmt *f, const fc *A, int32_t *x) {
  const int32_t s04 = sat(f, A[0].re + A[4].re), d04 = sat(f, A[0].re - A[4].re);
  const int32_t s26 = sat(f, A[2].re + A[6].re), e26 = sat(f, A[2].im - A[6].im);
  const fc p15 = {sat(f, A[1].re - A[5].re), sat(f, A[1].im - A[5].im)};
  const fc p37 = {sat(f, A[3].re - A[7].re), sat(f, A[3].im - A[7].im)};
  const int32_t qr = sat(f, sat(f, A[1].re + A[5].re) + sat(f, A[3].re + A[7].re));
  const int32_t qi = sat(f, sat(f, A[1].im + A[5].im) - sat(f, A[3].im + A[7].im));
  const int32_t u = rdm(f, sat(f, p15.re - p37.re), f->c8); /* c8 (a - b), one rounding */
  const int32_t v = rdm(f, sat(f, p15.im + p37.im), f->c8);
  const int32_t e = sat(f, s04 + s26), g = sat(f, s04 - s26);
  const int32_t a = sat(f, d04 + u), b = sat(f, sat(f, -(int64_t)e26) - v);
  const int32_t c = sat(f, d04 - u), d = sat(f, v - e26);
  x[0] = sat(f, e + qr);
  x[4] = sat(f, e - qr);
  x[2] = sat(f, g - qi);
  x[6] = sat(f, g + qi);
  x[1] = sat(f, a + b);
  x[7] = sat(f, a - b);
  x[3] = sat(f, c - d);
  x[5] = sat(f, c + d);
}

/* real-output codelet of length 16 on the extended, pre-shifted inputs A:
 * the split-radix real parts; the odd quarter-wave terms are rotated by
 * pairs of two-product MACs, the eighth-wave terms by a rounded c8 product
 * folded into a MAC with the unit constant */
static void real_out16(const fmt *f, const fc *A, int32_t *x) {
#define SA(a, b) sat(f, (int64_t)(a) + (b))
#define SS(a, b) sat(f, (int64_t)(a) - (b))
  const int32_t C8 = f->c8, C16 = f->c16, S16 = f->s16, HI = f->one, LO = f->mone;
  /* even half: inputs 0, 2, ..., 14 */
  const int32_t s08 = SA(A[0].re, A[8].re), d08 = SS(A[0].re, A[8].re);
  const int32_t s4c = SA(A[4].re, A[12].re), d4c = SS(A[4].im, A[12].im);
  const int32_t ev = SA(s08, s4c), ew = SS(s08, s4c);
  const int32_t s2a6e = SA(SA(A[2].re, A[10].re), SA(A[6].re, A[14].re));
  const int32_t r2a = SS(A[2].re, A[10].re), i2a = SS(A[2].im, A[10].im);
  const int32_t r6e = SS(A[6].re, A[14].re), i6e = SS(A[6].im, A[14].im);
  const int32_t i26 = SS(SA(A[2].im, A[10].im), SA(A[6].im, A[14].im));
  const int32_t e0 = SA(ev, s2a6e), e4 = SS(ev, s2a6e);
  const int32_t f1 = SS(d08, d4c), f3 = SA(d08, d4c);
  const int32_t f2 = SS(ew, i26), f6 = SA(ew, i26);
  /* odd half: inputs 1, 3, ..., 15 */
  const int32_t s19 = SA(A[1].re, A[9].re), s5d = SA(A[5].re, A[13].re);
  const int32_t s3b = SA(A[3].re, A[11].re), s7f = SA(A[7].re, A[15].re);
  const int32_t o0 = SA(SA(s19, s5d), SA(s3b, s7f));
  const int32_t i3b = SS(A[3].im, A[11].im), r7f = rdm(f, SS(A[7].re, A[15].re), HI);
  const int32_t r3b = SS(A[3].re, A[11].re), i7f = rdm(f, SS(A[7].im, A[15].im), LO);
  const int32_t i19 = SS(A[1].im, A[9].im), r5d = rdm(f, SS(A[5].re, A[13].re), HI);
  const int32_t r19 = SS(A[1].re, A[9].re), i5d = rdm(f, SS(A[5].im, A[13].im), LO);
  const int32_t p3 = SA(i3b, r7f), q3 = SA(r3b, i7f), p1 = SA(i19, r5d), q1 = SA(r19, i5d);
  const int32_t m3 = SS(i3b, r7f), n3 = SS(r3b, i7f), m1 = SS(i19, r5d), n1 = SS(r19, i5d);
  const int32_t j3b = SA(A[3].im, A[11].im), j7f = SA(A[7].im, A[15].im), j37 = SS(j3b, j7f);
  const int32_t k37 = SS(s3b, s7f);
  const int32_t j19 = SA(A[1].im, A[9].im), j5d = SA(A[5].im, A[13].im), j15 = SS(j19, j5d);
  const int32_t k15 = SS(s19, s5d);
  const int32_t o4 = SS(SA(j19, j5d), SA(j3b, j7f));
  /* rotations */
  const int32_t w1 = rdm(f, SS(mac2(f, i6e, -C8, rdm(f, r6e, -C8), HI), mac2(f, i2a, C8, rdm(f, r2a, C8), LO)), LO);
  const int32_t w3 = SA(mac2(f, r2a, C8, rdm(f, i2a, C8), HI), mac2(f, r6e, -C8, rdm(f, i6e, -C8), LO));
  const int32_t z2 = rdm(f, SS(mac2(f, j37, -C8, rdm(f, k37, -C8), HI), mac2(f, j15, C8, rdm(f, k15, C8), LO)), LO);
  const int32_t z6 = SA(mac2(f, k15, C8, rdm(f, j15, C8), HI), mac2(f, k37, -C8, rdm(f, j37, -C8), LO));
  const int32_t z1 = rdm(f, SS(mac2(f, p3, -C16, q3, S16), mac2(f, p1, S16, q1, -C16)), LO);
  const int32_t z3 = rdm(f, SS(mac2(f, m3, S16, n3, -C16), mac2(f, m1, C16, n1, -S16)), LO);
  const int32_t z5 = SA(mac2(f, q1, S16, p1, C16), mac2(f, q3, -C16, p3, -S16));
  const int32_t z7 = SA(mac2(f, n1, C16, m1, S16), mac2(f, n3, S16, m3, C16));
  const int32_t g1 = SS(f1, w1), g5 = SA(f1, w1), g3 = SS(f3, w3), g7 = SA(f3, w3);
  x[0] = SA(e0, o0);
  x[8] = SS(e0, o0);
  x[4] = SS(e4, o4);
  x[12] = SA(e4, o4);
  x[2] = SS(f2, z2);
  x[10] = SA(f2, z2);
  x[6] = SS(f6, z6);
  x[14] = SA(f6, z6);
  x[1] = SS(g1, z1);
  x[9] = SA(g1, z1);
  x[3] = SS(g3, z3);
  x[11] = SA(g3, z3);
  x[5] = SS(g5, z5);
  x[13] = SA(g5, z5);
  x[7] = SS(g7, z7);
  x[15] = SA(g7, z7);
#undef SA
#undef SS
}

/* real-output codelet of length r (2..16) over the Hermitian half
 * X[e * xs], e = 0..r/2 */
static void real_out(const fmt *f, int r, const fc *X, int64_t xs, int32_t *x) {
  const int s = ilog2(r);
  fc A[16] = {{0, 0}}, y[16];
  for (int i = 0; i < r; ++i) A[i] = i <= r / 2 ? cx_in(f, X[i * xs], s, 0) : cx_in(f, X[(r - i) * xs], s, 1);
  if (r == 8) {
    real_out8(f, A, x);
  } else if (r == 16) {
    real_out16(f, A, x);
  } else {
    codelet(f, r, 1, A, y);
    for (int k = 0; k < r; ++k) x[k] = y[k].re;
  }
}

/* row j of a radix-16 DIF level over `rows` rows of a Hermitian sequence
 * of length 16 rows (stored half X[e * xs], e = 0..8 rows): the 16 outputs,
 * twiddled by W_{16 rows}^{jk} (w: the backward table over `rows` rows) */
static void dif_row(const fmt *f, const fc *X, int64_t xs, int64_t rows, int64_t j, const int32_t *w, fc *y) {
  fc a[16], t[16];
  for (int i = 0; i < 16; ++i) {
    const int direct = j == 0 ? i <= 8 : i <= 7;
    a[i] = direct ? cx_in(f, X[(j + rows * i) * xs], 4, 0) : cx_in(f, X[(rows * (16 - i) - j) * xs], 4, 1);
  }
  codelet(f, 16, 1, a, t);
  for (int k = 0; k < 16; ++k) {
    if (j > 0 && k > 0) {
      const int32_t *c = w + 4 * (15 * (j - 1) + (k - 1));
      y[k] = (fc){mac2(f, t[k].re, c[0], t[k].im, c[2]), mac2(f, t[k].re, c[1], t[k].im, c[3])};
    } else {
      y[k] = t[k];
    }
  }
}

/* fixed-point C2R (backward) of power-of-two n in [2, 4096]: inputs bins
 * 0..n/2 (istride / idist in complex elements), outputs n reals (ostride /
 * odist in reals), scaled by 1/n */
static int fixed_c2r(int bits, const void *in, void *out, int64_t n, int64_t howmany, int64_t istride,
                     int64_t idist, int64_t ostride, int64_t odist) {
  if (n < 2 || n > 4096 || (n & (n - 1))) return -1;
  const fmt F = make_fmt(bits), *f = &F;
  const size_t esz = (size_t)(bits / 4), rsz = (size_t)(bits / 8);
  const int64_t h = n / 2 + 1, m = n / 16, m2 = n > 256 ? n / 256 : 0;
  int32_t *w = NULL, *w2 = NULL;
  if (n > 16) {
    w = (int32_t *)malloc(sizeof(int32_t) * 4 * 15 * (size_t)(m > 1 ? m - 1 : 1));
    twiddles16(f, m, 1, w);
  }
  if (m2) {
    w2 = (int32_t *)malloc(sizeof(int32_t) * 4 * 15 * (size_t)(m2 > 1 ? m2 - 1 : 1));
    twiddles16(f, m2, 1, w2);
  }
#pragma omp parallel
  {
  fc *X = (fc *)malloc(sizeof(fc) * (size_t)h); /* per-thread scratch */
  fc *b = (fc *)malloc(sizeof(fc) * (size_t)n);
  fc *c = (fc *)malloc(sizeof(fc) * (size_t)n);
  int32_t *x = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
#pragma omp for schedule(static)
  for (int64_t mb = 0; mb < howmany; ++mb) {
    for (int64_t k = 0; k < h; ++k) X[k] = ld(bits, (const char *)in + esz * (size_t)(mb * idist + k * istride), 0);
    if (n <= 16) {
      real_out(f, (int)n, X, 1, x);
    } else {
      for (int64_t j = 0; j <= m / 2; ++j) dif_row(f, X, 1, m, j, w, b + 16 * j);
      if (!m2) {
        for (int k = 0; k < 16; ++k) {
          int32_t col[16];
          real_out(f, (int)m, b + k, 16, col);
          for (int64_t t = 0; t < m; ++t) x[k + 16 * t] = col[t];
        }
      } else {
        for (int k = 0; k < 16; ++k)
          for (int64_t i = 0; i <= m2 / 2; ++i) {
            fc y[16];
            dif_row(f, b + k, 16, m2, i, w2, y);
            for (int q = 0; q < 16; ++q) c[256 * i + 16 * q + k] = y[q];
          }
        for (int l = 0; l < 256; ++l) {
          int32_t col[16];
          real_out(f, (int)m2, c + l, 256, col);
          for (int64_t t = 0; t < m2; ++t) x[l + 256 * t] = col[t];
        }
      }
    }
    for (int64_t t = 0; t < n; ++t) {
      char *p = (char *)out + rsz * (size_t)(mb * odist + t * ostride);
      if (bits == 16)
        *(int16_t *)p = (int16_t)x[t];
      else
        *(int8_t *)p = (int8_t)x[t];
    }
  }
  free(X);
  free(b);
  free(c);
  free(x);
  }
  free(w);
  free(w2);
  return 0;
}

int oracle_q15_c2r(const int16_t *in, int16_t *out, int64_t n, int64_t howmany, int64_t istride, int64_t idist,
                   int64_t ostride, int64_t odist) {
  return fixed_c2r(16, in, out, n, howmany, istride, idist, ostride, odist);
}

int oracle_q7_c2r(const int8_t *in, int8_t *out, int64_t n, int64_t howmany, int64_t istride, int64_t idist,
                  int64_t ostride, int64_t odist) {
  return fixed_c2r(8, in, out, n, howmany, istride, idist, ostride, odist);
}

int oracle_q15_r2c(const int16_t *in, int16_t *out, int64_t n, int64_t howmany, int64_t istride, int64_t idist,
                   int64_t ostride, int64_t odist) {
  return fixed_r2c(16, in, out, n, howmany, istride, idist, ostride, odist);
}

int oracle_q7_r2c(const int8_t *in, int8_t *out, int64_t n, int64_t howmany, int64_t istride, int64_t idist,
                  int64_t ostride, int64_t odist) {
  return fixed_r2c(8, in, out, n, howmany, istride, idist, ostride, odist);
}

int oracle_q15_c2c(const int16_t *in, int16_t *out, int64_t n, int64_t howmany, int64_t idist, int64_t odist,
                   int dir) {
  return fixed_c2c(16, in, out, n, howmany, idist, odist, dir);
}

int oracle_q7_c2c(const int8_t *in, int8_t *out, int64_t n, int64_t howmany, int64_t idist, int64_t odist,
                  int dir) {
  return fixed_c2c(8, in, out, n, howmany, idist, odist, dir);
}

/* the outer radix-16 level's Q0.15 twiddle table for length n (n / 16 rows),
 * as int16: (c, s, cvt(-s), c) per (row, input) */
void oracle_q15_twiddles(int64_t n, int dir, int16_t *w) {
  const fmt F = make_fmt(16);
  const int64_t m = n / 16;
  int32_t *t = (int32_t *)malloc(sizeof(int32_t) * 4 * 15 * (size_t)(m > 1 ? m - 1 : 1));
  twiddles16(&F, m, dir, t);
  for (int64_t i = 0; i < 4 * 15 * (m - 1); ++i) w[i] = (int16_t)t[i];
  free(t);
}
