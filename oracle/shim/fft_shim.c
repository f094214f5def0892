/* FP64 mixed-radix Stockham FFT serving the FFTW3 entry points the reference calls.
 *
 * Test infrastructure only (CPU oracle build of the reference, CPU FFT checker for the tests).
 * Conventions follow FFTW3's documented ones, which the reference relies on in
 * src/fftw_helper.cpp:5-33 (forward = sign -1, backward = sign +1, both unnormalised; the
 * reference divides by N itself) and src/solver.cpp:1439-1440 (2D plans, row-major n0 x n1).
 *
 * Algorithm: self-sorting Stockham decimation-in-time, radix 4/2/3/5 butterflies plus a plain DFT
 * for any other prime factor.  Stage s with radix p, l = product of earlier radices, r = n/(l p):
 *   a_q = x[j r p + q r + k] * w_{l p}^{j q},   y[(j + t l) r + k] = sum_q a_q w_p^{q t}.
 * Twiddles come from one table of n roots computed with sin/cos of 2 pi m / n.
 * Not thread-safe (the 1D plan cache owns its work buffers); the reference is single-threaded. */
#include "fftw3.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct fft1d {
  int n, sign, nstage;
  int radix[40];
  double* roots;   /* 2n doubles: exp(sign 2 pi i m / n) */
  double* tw[40];  /* per stage: l*(p-1) complex twiddles */
  double* work;    /* 2n doubles ping-pong buffer */
  double* col;     /* 2n doubles column gather buffer */
  struct fft1d* next;
} fft1d;

struct oracle_fft_plan {
  int n0, n1, sign;
  double* in;
  double* out;
  fft1d* p0;
  fft1d* p1;
};

static fft1d* g_cache = NULL;

static fft1d* fft1d_get(int n, int sign) {
  for (fft1d* p = g_cache; p; p = p->next)
    if (p->n == n && p->sign == sign) return p;
  fft1d* p = (fft1d*)calloc(1, sizeof(fft1d));
  p->n = n;
  p->sign = sign;
  int m = n;
  while (m % 4 == 0 && m > 4) { p->radix[p->nstage++] = 4; m /= 4; }
  if (m % 4 == 0) { p->radix[p->nstage++] = 4; m /= 4; }
  while (m % 2 == 0) { p->radix[p->nstage++] = 2; m /= 2; }
  while (m % 3 == 0) { p->radix[p->nstage++] = 3; m /= 3; }
  while (m % 5 == 0) { p->radix[p->nstage++] = 5; m /= 5; }
  for (int f = 7; m > 1; f += 2)
    while (m % f == 0) { p->radix[p->nstage++] = f; m /= f; }
  for (int s = 0; s < p->nstage; ++s)
    if (p->radix[s] > 256) abort(); /* prime factors above 256 are not supported */
  p->roots = (double*)malloc(sizeof(double) * 2 * (size_t)n);
  for (int k = 0; k < n; ++k) {
    double a = 2.0 * M_PI * (double)k / (double)n;
    p->roots[2 * k] = cos(a);
    p->roots[2 * k + 1] = (double)sign * sin(a);
  }
  int l = 1;
  for (int s = 0; s < p->nstage; ++s) {
    int r = p->radix[s];
    int L = l * r;
    p->tw[s] = (double*)malloc(sizeof(double) * 2 * (size_t)(l * (r - 1) + 1));
    for (int j = 0; j < l; ++j)
      for (int q = 1; q < r; ++q) {
        long idx = ((long)j * q * (n / L)) % n;
        p->tw[s][2 * (j * (r - 1) + q - 1)] = p->roots[2 * idx];
        p->tw[s][2 * (j * (r - 1) + q - 1) + 1] = p->roots[2 * idx + 1];
      }
    l = L;
  }
  p->work = (double*)malloc(sizeof(double) * 2 * (size_t)n);
  p->col = (double*)malloc(sizeof(double) * 2 * (size_t)n);
  p->next = g_cache;
  g_cache = p;
  return p;
}

/* One Stockham pass: x (r p) x l -> y r x (l p). */
static void stage(const fft1d* P, int s, int l, const double* x, double* y) {
  const int n = P->n, p = P->radix[s], r = n / (l * p);
  const double sg = (double)P->sign;
  const double* tw = P->tw[s];
  double ar[256], ai[256]; /* radices above 256 are rejected in fft1d_get */
  for (int j = 0; j < l; ++j) {
    const double* w = tw + 2 * j * (p - 1);
    for (int k = 0; k < r; ++k) {
      const double* src = x + 2 * ((long)j * r * p + k);
      ar[0] = src[0];
      ai[0] = src[1];
      for (int q = 1; q < p; ++q) {
        double xr = src[2 * q * r], xi = src[2 * q * r + 1];
        double wr = w[2 * (q - 1)], wi = w[2 * (q - 1) + 1];
        ar[q] = xr * wr - xi * wi;
        ai[q] = xr * wi + xi * wr;
      }
      double* dst = y + 2 * ((long)j * r + k);
      const long so = 2L * l * r; /* output stride between t and t+1 */
      if (p == 2) {
        dst[0] = ar[0] + ar[1]; dst[1] = ai[0] + ai[1];
        dst[so] = ar[0] - ar[1]; dst[so + 1] = ai[0] - ai[1];
      } else if (p == 4) {
        double s0r = ar[0] + ar[2], s0i = ai[0] + ai[2];
        double d0r = ar[0] - ar[2], d0i = ai[0] - ai[2];
        double s1r = ar[1] + ar[3], s1i = ai[1] + ai[3];
        double d1r = ar[1] - ar[3], d1i = ai[1] - ai[3];
        /* w4 * (d1) with w4 = sign * i */
        double er = -sg * d1i, ei = sg * d1r;
        dst[0] = s0r + s1r; dst[1] = s0i + s1i;
        dst[so] = d0r + er; dst[so + 1] = d0i + ei;
        dst[2 * so] = s0r - s1r; dst[2 * so + 1] = s0i - s1i;
        dst[3 * so] = d0r - er; dst[3 * so + 1] = d0i - ei;
      } else if (p == 3) {
        const double h = 0.86602540378443864676; /* sqrt(3)/2 */
        double tr = ar[1] + ar[2], ti = ai[1] + ai[2];
        double mr = ar[0] - 0.5 * tr, mi = ai[0] - 0.5 * ti;
        double dr = sg * h * (ar[1] - ar[2]), di = sg * h * (ai[1] - ai[2]);
        dst[0] = ar[0] + tr; dst[1] = ai[0] + ti;
        dst[so] = mr - di; dst[so + 1] = mi + dr;
        dst[2 * so] = mr + di; dst[2 * so + 1] = mi - dr;
      } else if (p == 5) {
        const double c1 = 0.30901699437494742410, c2 = -0.80901699437494742410;
        const double s1 = 0.95105651629515357212, s2 = 0.58778525229247312917;
        double t1r = ar[1] + ar[4], t1i = ai[1] + ai[4];
        double t2r = ar[2] + ar[3], t2i = ai[2] + ai[3];
        double t3r = ar[1] - ar[4], t3i = ai[1] - ai[4];
        double t4r = ar[2] - ar[3], t4i = ai[2] - ai[3];
        double m1r = ar[0] + c1 * t1r + c2 * t2r, m1i = ai[0] + c1 * t1i + c2 * t2i;
        double m2r = ar[0] + c2 * t1r + c1 * t2r, m2i = ai[0] + c2 * t1i + c1 * t2i;
        double u1r = sg * (s1 * t3r + s2 * t4r), u1i = sg * (s1 * t3i + s2 * t4i);
        double u2r = sg * (s2 * t3r - s1 * t4r), u2i = sg * (s2 * t3i - s1 * t4i);
        dst[0] = ar[0] + t1r + t2r; dst[1] = ai[0] + t1i + t2i;
        dst[so] = m1r - u1i; dst[so + 1] = m1i + u1r;
        dst[4 * so] = m1r + u1i; dst[4 * so + 1] = m1i - u1r;
        dst[2 * so] = m2r - u2i; dst[2 * so + 1] = m2i + u2r;
        dst[3 * so] = m2r + u2i; dst[3 * so + 1] = m2i - u2r;
      } else {
        const int step = n / p;
        for (int t = 0; t < p; ++t) {
          double br = 0.0, bi = 0.0;
          for (int q = 0; q < p; ++q) {
            long m = ((long)q * t) % p;
            double wr = P->roots[2 * m * step], wi = P->roots[2 * m * step + 1];
            br += ar[q] * wr - ai[q] * wi;
            bi += ar[q] * wi + ai[q] * wr;
          }
          dst[t * so] = br;
          dst[t * so + 1] = bi;
        }
      }
    }
  }
}

/* Transform src (contiguous, n complex) into dst; src is left intact unless src == dst. */
static void fft1d_exec(const fft1d* P, const double* src, double* dst) {
  const int n = P->n;
  if (src == dst) { /* in place: stage the input in a private copy */
    memcpy(P->col, src, sizeof(double) * 2 * (size_t)n);
    src = P->col;
  }
  if (P->nstage == 0) {
    if (dst != src) memcpy(dst, src, sizeof(double) * 2 * (size_t)n);
    return;
  }
  /* Ping-pong between dst and work so that the last stage lands in dst. */
  double* bufs[2];
  if ((P->nstage % 2) == 1) { bufs[0] = dst; bufs[1] = P->work; }
  else { bufs[0] = P->work; bufs[1] = dst; }
  const double* x = src;
  int l = 1;
  for (int s = 0; s < P->nstage; ++s) {
    double* y = bufs[s % 2];
    stage(P, s, l, x, y);
    x = y;
    l *= P->radix[s];
  }
}

static void fft2d_exec(fft1d* p0, fft1d* p1, int n0, int n1, const double* in, double* out) {
  for (int i = 0; i < n0; ++i) fft1d_exec(p1, in + 2L * i * n1, out + 2L * i * n1);
  if (n0 == 1) return;
  double* colin = (double*)malloc(sizeof(double) * 2 * (size_t)n0);
  double* colout = (double*)malloc(sizeof(double) * 2 * (size_t)n0);
  for (int c = 0; c < n1; ++c) {
    for (int i = 0; i < n0; ++i) {
      colin[2 * i] = out[2 * ((long)i * n1 + c)];
      colin[2 * i + 1] = out[2 * ((long)i * n1 + c) + 1];
    }
    fft1d_exec(p0, colin, colout);
    for (int i = 0; i < n0; ++i) {
      out[2 * ((long)i * n1 + c)] = colout[2 * i];
      out[2 * ((long)i * n1 + c) + 1] = colout[2 * i + 1];
    }
  }
  free(colin);
  free(colout);
}

fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex* in, fftw_complex* out, int sign, unsigned flags) {
  (void)flags;
  struct oracle_fft_plan* p = (struct oracle_fft_plan*)malloc(sizeof(struct oracle_fft_plan));
  p->n0 = n0;
  p->n1 = n1;
  p->sign = sign;
  p->in = (double*)in;
  p->out = (double*)out;
  p->p0 = fft1d_get(n0, sign);
  p->p1 = fft1d_get(n1, sign);
  return p;
}

void fftw_execute(const fftw_plan p) { fft2d_exec(p->p0, p->p1, p->n0, p->n1, p->in, p->out); }

void fftw_destroy_plan(fftw_plan p) { free(p); }

void* fftw_malloc(size_t n) {
  void* ptr = NULL;
  if (posix_memalign(&ptr, 64, n ? n : 64) != 0) return NULL;
  return ptr;
}

void fftw_free(void* p) { free(p); }

void oracle_fft2d(int n0, int n1, double* data, int sign) {
  fft2d_exec(fft1d_get(n0, sign), fft1d_get(n1, sign), n0, n1, data, data);
}
