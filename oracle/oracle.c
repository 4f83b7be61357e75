/*
 * FP64 CPU oracle for the batched 1D transforms -- TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load this library, and only to check results.  The product path
 * (libplfft_b200.so) never calls it.
 *
 * Conventions restated from the reference (arm/perf-libs-fft):
 *   docs/plfft.md:100-116   forward X[k] = sum_j x[j] e^{-2 pi i jk/n},
 *                           backward with +; R2C keeps bins 0..n/2, C2R reads
 *                           them and fills the rest by conjugate symmetry
 *   docs/plfft.md:121-134   float transforms unnormalized
 *   docs/plfft.md:140-166   element b,k at ptr[b*dist + k*stride]
 *   include/plfft.h:98-134, docs/plfft.md:186-212
 *                           R2R kinds = FFTW REDFT00/10/01/11, RODFT00/10/01/
 *                           11, DHT, R2HC/HC2R (half-complex order)
 *
 * Two DFT evaluators:
 *   oracle_dft_*  direct O(n^2) sums with exactly reduced twiddle indices
 *                 (j*k mod n), the ground truth for n up to ~2^14;
 *   oracle_fft_*  recursive mixed-radix Cooley-Tukey in FP64 (prime factors
 *                 <= 64 by direct DFT, larger ones by FP64 Bluestein), for
 *                 large n; itself checked against oracle_dft_* by the tests.
 *
 * Data: complex values are interleaved (re, im) doubles.  Batch loops are
 * OpenMP-parallel over members with `threads` threads (0 = runtime default).
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* cos/sin of 2 pi k / n with exact integer reduction of the angle */
static void root(int64_t k, int64_t n, double *c, double *s) {
  k %= n;
  if (k < 0) k += n;
  /* angle = 2 pi k/n; fold into [0, pi/4] by octant */
  __int128 k8 = (__int128)8 * k;
  int64_t oct = (int64_t)(k8 / n);
  int64_t rem = (int64_t)(k8 - (__int128)oct * n);
  long double r = (long double)rem / (long double)n * (3.141592653589793238462643383279502884L / 4.0L);
  long double c0, s0;
  if (oct % 2 == 0) {
    c0 = cosl(r);
    s0 = sinl(r);
  } else {
    long double r2 = 3.141592653589793238462643383279502884L / 4.0L - r;
    c0 = cosl(r2);
    s0 = -sinl(r2);
    oct += 1;
  }
  int64_t q = (oct / 2) % 4;
  long double cc = c0, ss = s0;
  if (q == 1) { cc = -s0; ss = c0; }
  if (q == 2) { cc = -c0; ss = -s0; }
  if (q == 3) { cc = s0; ss = -c0; }
  *c = (double)cc;
  *s = (double)ss;
}

/* table of e^{sign 2 pi i k/n}, k < n */
static double *root_table(int64_t n, int sign) {
  double *t = (double *)malloc(sizeof(double) * 2 * (size_t)n);
  for (int64_t k = 0; k < n; ++k) {
    double c, s;
    root(k, n, &c, &s);
    t[2 * k] = c;
    t[2 * k + 1] = sign * s;
  }
  return t;
}

/* ------------------------------------------------------------------------ */
/* direct DFT of one contiguous complex vector                              */
/* ------------------------------------------------------------------------ */
static void dft1(const double *x, double *y, int64_t n, const double *w) {
  for (int64_t k = 0; k < n; ++k) {
    long double re = 0, im = 0;
    int64_t idx = 0;
    for (int64_t j = 0; j < n; ++j) {
      const double a = x[2 * j], b = x[2 * j + 1];
      const double c = w[2 * idx], s = w[2 * idx + 1];
      re += (long double)a * c - (long double)b * s;
      im += (long double)a * s + (long double)b * c;
      idx += k;
      if (idx >= n) idx -= n;
    }
    y[2 * k] = (double)re;
    y[2 * k + 1] = (double)im;
  }
}

/* ------------------------------------------------------------------------ */
/* FP64 FFT (any n)                                                          */
/* ------------------------------------------------------------------------ */
static int64_t smallest_factor(int64_t n) {
  for (int64_t p = 2; p * p <= n; ++p)
    if (n % p == 0) return p;
  return n;
}

/* Recursive FFT state: W = table of e^{sign 2 pi i k / N} for the top-level
 * length N; every sub-length n divides N, so W_n^e = W[e * (N/n) mod N]. */
typedef struct {
  const double *w;
  int64_t big;
  int sign;
} fft_ctx;

static void fft_rec(const fft_ctx *cx, const double *x, int64_t xs, double *y, int64_t n, double *scratch);
static void fft_vec(const double *x, double *y, int64_t n, int sign);

/* Bluestein in FP64 for a large prime n, pad to a power of two */
static void bluestein(const double *x, int64_t xs, double *y, int64_t n, int sign) {
  int64_t m = 1;
  while (m < 2 * n - 1) m <<= 1;
  double *a = (double *)calloc(2 * (size_t)m, sizeof(double));
  double *b = (double *)calloc(2 * (size_t)m, sizeof(double));
  double *A = (double *)malloc(sizeof(double) * 2 * (size_t)m);
  double *B = (double *)malloc(sizeof(double) * 2 * (size_t)m);
  double *w = (double *)malloc(sizeof(double) * 2 * (size_t)n);
  for (int64_t k = 0; k < n; ++k) {
    /* w_k = e^{sign i pi k^2 / n}, k^2 mod 2n in integers */
    int64_t e = (int64_t)(((__int128)k * k) % (2 * n));
    double c, s;
    root(e, 2 * n, &c, &s);
    w[2 * k] = c;
    w[2 * k + 1] = sign * s;
  }
  for (int64_t k = 0; k < n; ++k) {
    const double xr = x[2 * k * xs], xi = x[2 * k * xs + 1];
    a[2 * k] = xr * w[2 * k] - xi * w[2 * k + 1];
    a[2 * k + 1] = xr * w[2 * k + 1] + xi * w[2 * k];
    b[2 * k] = w[2 * k];
    b[2 * k + 1] = -w[2 * k + 1];
    if (k) {
      b[2 * (m - k)] = w[2 * k];
      b[2 * (m - k) + 1] = -w[2 * k + 1];
    }
  }
  fft_vec(a, A, m, -1);
  fft_vec(b, B, m, -1);
  for (int64_t k = 0; k < m; ++k) {
    const double ar = A[2 * k], ai = A[2 * k + 1], br = B[2 * k], bi = B[2 * k + 1];
    A[2 * k] = ar * br - ai * bi;
    A[2 * k + 1] = ar * bi + ai * br;
  }
  fft_vec(A, a, m, +1);
  for (int64_t k = 0; k < n; ++k) {
    const double cr = a[2 * k] / m, ci = a[2 * k + 1] / m;
    y[2 * k] = cr * w[2 * k] - ci * w[2 * k + 1];
    y[2 * k + 1] = cr * w[2 * k + 1] + ci * w[2 * k];
  }
  free(a); free(b); free(A); free(B); free(w);
}

static inline void wget(const fft_ctx *cx, int64_t e, int64_t n, double *c, double *s) {
  const int64_t idx = (int64_t)(((__int128)e * (cx->big / n)) % cx->big);
  *c = cx->w[2 * idx];
  *s = cx->w[2 * idx + 1];
}

/* y[0..n) = DFT of x[0], x[xs], ... ; scratch holds >= 4n complex */
static void fft_rec(const fft_ctx *cx, const double *x, int64_t xs, double *y, int64_t n, double *scratch) {
  if (n == 1) {
    y[0] = x[0];
    y[1] = x[1];
    return;
  }
  const int64_t p = smallest_factor(n);
  if (p == n && n > 64) {
    bluestein(x, xs, y, n, cx->sign);
    return;
  }
  if (p == n) {
    for (int64_t k = 0; k < n; ++k) {
      double re = 0, im = 0;
      int64_t idx = 0;
      for (int64_t j = 0; j < n; ++j) {
        double c, s;
        wget(cx, idx, n, &c, &s);
        const double a = x[2 * j * xs], b = x[2 * j * xs + 1];
        re += a * c - b * s;
        im += a * s + b * c;
        idx += k;
        if (idx >= n) idx -= n;
      }
      y[2 * k] = (double)re;
      y[2 * k + 1] = (double)im;
    }
    return;
  }
  /* decimation in time: n = p * m, sub-transforms of x[p*j + r] */
  const int64_t m = n / p;
  double *sub = scratch; /* p sub-results of length m, contiguous */
  double *scr2 = scratch + 2 * n;
  for (int64_t r = 0; r < p; ++r) fft_rec(cx, x + 2 * r * xs, xs * p, sub + 2 * r * m, m, scr2);
  /* combine: y[k + m q] = sum_r W_n^{r(k + m q)} sub_r[k] */
  double tbuf[2 * 64];
  double *t = p <= 64 ? tbuf : (double *)malloc(sizeof(double) * 2 * (size_t)p);
  for (int64_t k = 0; k < m; ++k) {
    for (int64_t r = 0; r < p; ++r) {
      double c, s;
      wget(cx, r * k, n, &c, &s);
      const double a = sub[2 * (r * m + k)], b = sub[2 * (r * m + k) + 1];
      t[2 * r] = a * c - b * s;
      t[2 * r + 1] = a * s + b * c;
    }
    for (int64_t q = 0; q < p; ++q) {
      double re = 0, im = 0;
      int64_t idx = 0;
      for (int64_t r = 0; r < p; ++r) {
        double c, s;
        wget(cx, idx, p, &c, &s);
        re += t[2 * r] * c - t[2 * r + 1] * s;
        im += t[2 * r] * s + t[2 * r + 1] * c;
        idx += q;
        if (idx >= p) idx -= p;
      }
      y[2 * (k + m * q)] = (double)re;
      y[2 * (k + m * q) + 1] = (double)im;
    }
  }
  if (t != tbuf) free(t);
}

static void fft_vec(const double *x, double *y, int64_t n, int sign) {
  double *scr = (double *)malloc(sizeof(double) * 8 * (size_t)(n + 64));
  double *w = root_table(n, sign);
  fft_ctx cx = {w, n, sign};
  fft_rec(&cx, x, 1, y, n, scr);
  free(w);
  free(scr);
}

static void dft_vec(const double *x, double *y, int64_t n, int sign) {
  double *w = root_table(n, sign);
  dft1(x, y, n, w);
  free(w);
}

typedef void (*vec_fn)(const double *, double *, int64_t, int);

static void set_threads(int threads) {
  if (threads > 0) omp_set_num_threads(threads);
}

/* ------------------------------------------------------------------------ */
/* public entry points (complex interleaved doubles, element strides)        */
/* ------------------------------------------------------------------------ */
static void c2c_batch(vec_fn f, const double *in, double *out, int64_t n, int64_t howmany, int64_t is,
                      int64_t id, int64_t os, int64_t od, int dir, int threads) {
  set_threads(threads);
#pragma omp parallel
  {
    double *x = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    double *y = (double *)malloc(sizeof(double) * 2 * (size_t)n);
#pragma omp for schedule(dynamic)
    for (int64_t b = 0; b < howmany; ++b) {
      for (int64_t j = 0; j < n; ++j) {
        x[2 * j] = in[2 * (b * id + j * is)];
        x[2 * j + 1] = in[2 * (b * id + j * is) + 1];
      }
      f(x, y, n, dir);
      for (int64_t k = 0; k < n; ++k) {
        out[2 * (b * od + k * os)] = y[2 * k];
        out[2 * (b * od + k * os) + 1] = y[2 * k + 1];
      }
    }
    free(x);
    free(y);
  }
}

void oracle_dft_c2c(const double *in, double *out, int64_t n, int64_t howmany, int64_t is, int64_t id,
                    int64_t os, int64_t od, int dir, int threads) {
  c2c_batch(dft_vec, in, out, n, howmany, is, id, os, od, dir, threads);
}

void oracle_fft_c2c(const double *in, double *out, int64_t n, int64_t howmany, int64_t is, int64_t id,
                    int64_t os, int64_t od, int dir, int threads) {
  c2c_batch(fft_vec, in, out, n, howmany, is, id, os, od, dir, threads);
}

/* R2C: real in (double), complex out bins 0..n/2 */
void oracle_r2c(const double *in, double *out, int64_t n, int64_t howmany, int64_t is, int64_t id,
                int64_t os, int64_t od, int use_fft, int threads) {
  set_threads(threads);
  const int64_t h = n / 2 + 1;
#pragma omp parallel
  {
    double *x = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    double *y = (double *)malloc(sizeof(double) * 2 * (size_t)n);
#pragma omp for schedule(dynamic)
    for (int64_t b = 0; b < howmany; ++b) {
      for (int64_t j = 0; j < n; ++j) {
        x[2 * j] = in[b * id + j * is];
        x[2 * j + 1] = 0.0;
      }
      (use_fft ? fft_vec : dft_vec)(x, y, n, -1);
      for (int64_t k = 0; k < h; ++k) {
        out[2 * (b * od + k * os)] = y[2 * k];
        out[2 * (b * od + k * os) + 1] = y[2 * k + 1];
      }
    }
    free(x);
    free(y);
  }
}

/* C2R: complex bins 0..n/2 in, real out; the imaginary parts of bin 0 and
 * (even n) bin n/2 are ignored, as a Hermitian spectrum implies */
void oracle_c2r(const double *in, double *out, int64_t n, int64_t howmany, int64_t is, int64_t id,
                int64_t os, int64_t od, int use_fft, int threads) {
  set_threads(threads);
  const int64_t h = n / 2 + 1;
#pragma omp parallel
  {
    double *x = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    double *y = (double *)malloc(sizeof(double) * 2 * (size_t)n);
#pragma omp for schedule(dynamic)
    for (int64_t b = 0; b < howmany; ++b) {
      for (int64_t k = 0; k < h; ++k) {
        x[2 * k] = in[2 * (b * id + k * is)];
        x[2 * k + 1] = in[2 * (b * id + k * is) + 1];
      }
      x[1] = 0.0;
      if (n % 2 == 0) x[2 * (n / 2) + 1] = 0.0;
      for (int64_t k = h; k < n; ++k) {
        x[2 * k] = x[2 * (n - k)];
        x[2 * k + 1] = -x[2 * (n - k) + 1];
      }
      (use_fft ? fft_vec : dft_vec)(x, y, n, +1);
      for (int64_t j = 0; j < n; ++j) out[b * od + j * os] = y[2 * j];
    }
    free(x);
    free(y);
  }
}

/* ------------------------------------------------------------------------ */
/* R2R kinds, direct sums of the FFTW definitions                            */
/* ------------------------------------------------------------------------ */
/* cos(pi * num / den) with num reduced mod 2 den in integers */
static double cospi_frac(int64_t num, int64_t den) {
  double c, s;
  root(num, 2 * den, &c, &s);
  return c;
}
static double sinpi_frac(int64_t num, int64_t den) {
  double c, s;
  root(num, 2 * den, &c, &s);
  return s;
}

static void r2r1(const double *x, double *y, int64_t n, int kind) {
  for (int64_t k = 0; k < n; ++k) {
    long double acc = 0;
    switch (kind) {
      case 0: /* DCT-I, REDFT00, n > 1: X0 + (-1)^k X_{n-1} + 2 sum_{j=1}^{n-2} X_j cos(pi jk/(n-1)) */
        acc = x[0] + ((k & 1) ? -x[n - 1] : x[n - 1]);
        for (int64_t j = 1; j < n - 1; ++j) acc += 2.0L * x[j] * cospi_frac(j * k, n - 1);
        break;
      case 1: /* DCT-II, REDFT10: 2 sum X_j cos(pi (2j+1) k / 2n) */
        for (int64_t j = 0; j < n; ++j) acc += 2.0L * x[j] * cospi_frac((2 * j + 1) * k, 2 * n);
        break;
      case 2: /* DCT-III, REDFT01: X0 + 2 sum_{j>=1} X_j cos(pi j (2k+1) / 2n) */
        acc = x[0];
        for (int64_t j = 1; j < n; ++j) acc += 2.0L * x[j] * cospi_frac(j * (2 * k + 1), 2 * n);
        break;
      case 3: /* DCT-IV, REDFT11: 2 sum X_j cos(pi (2j+1)(2k+1) / 4n) */
        for (int64_t j = 0; j < n; ++j) acc += 2.0L * x[j] * cospi_frac((2 * j + 1) * (2 * k + 1), 4 * n);
        break;
      case 4: /* DST-I, RODFT00: 2 sum X_j sin(pi (j+1)(k+1) / (n+1)) */
        for (int64_t j = 0; j < n; ++j) acc += 2.0L * x[j] * sinpi_frac((j + 1) * (k + 1), n + 1);
        break;
      case 5: /* DST-II, RODFT10: 2 sum X_j sin(pi (2j+1)(k+1) / 2n) */
        for (int64_t j = 0; j < n; ++j) acc += 2.0L * x[j] * sinpi_frac((2 * j + 1) * (k + 1), 2 * n);
        break;
      case 6: /* DST-III, RODFT01: (-1)^k X_{n-1} + 2 sum_{j<n-1} X_j sin(pi (j+1)(2k+1) / 2n) */
        acc = (k & 1) ? -x[n - 1] : x[n - 1];
        for (int64_t j = 0; j < n - 1; ++j) acc += 2.0L * x[j] * sinpi_frac((j + 1) * (2 * k + 1), 2 * n);
        break;
      case 7: /* DST-IV, RODFT11: 2 sum X_j sin(pi (2j+1)(2k+1) / 4n) */
        for (int64_t j = 0; j < n; ++j) acc += 2.0L * x[j] * sinpi_frac((2 * j + 1) * (2 * k + 1), 4 * n);
        break;
      case 8: /* DHT: sum X_j (cos + sin)(2 pi jk/n) */
        for (int64_t j = 0; j < n; ++j) {
          double c, s;
          root(j * k, n, &c, &s);
          acc += (long double)x[j] * (c + s);
        }
        break;
      case 9: { /* R2HC: r_k = Re F_k (k <= n/2), r_{n-k} = Im F_k (0 < k < (n+1)/2) */
        const int64_t kk = (k <= n / 2) ? k : n - k;
        long double re = 0, im = 0;
        for (int64_t j = 0; j < n; ++j) {
          double c, s;
          root(j * kk, n, &c, &s);
          re += (long double)x[j] * c;
          im -= (long double)x[j] * s;
        }
        acc = (k <= n / 2) ? re : im;
        break;
      }
      case 10: { /* HC2R: y_j = sum_k F_k e^{+2 pi i jk/n} with F from half-complex */
        const int64_t j = k;
        acc = x[0];
        for (int64_t m = 1; m < (n + 1) / 2; ++m) {
          double c, s;
          root(j * m, n, &c, &s);
          acc += 2.0L * ((long double)x[m] * c - (long double)x[n - m] * s);
        }
        if (n % 2 == 0) acc += (long double)x[n / 2] * ((j & 1) ? -1.0L : 1.0L);
        break;
      }
    }
    y[k] = (double)acc;
  }
}

void oracle_r2r(const double *in, double *out, int64_t n, int64_t howmany, int64_t is, int64_t id,
                int64_t os, int64_t od, int kind, int threads) {
  set_threads(threads);
#pragma omp parallel
  {
    double *x = (double *)malloc(sizeof(double) * (size_t)n);
    double *y = (double *)malloc(sizeof(double) * (size_t)n);
#pragma omp for schedule(dynamic)
    for (int64_t b = 0; b < howmany; ++b) {
      for (int64_t j = 0; j < n; ++j) x[j] = in[b * id + j * is];
      r2r1(x, y, n, kind);
      for (int64_t k = 0; k < n; ++k) out[b * od + k * os] = y[k];
    }
    free(x);
    free(y);
  }
}

int oracle_max_threads(void) { return omp_get_max_threads(); }
