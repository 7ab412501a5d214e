/*
 * fft64.h -- FP64 complex FFT (Stockham auto-sort, mixed radix, any length)
 * and a DCT-II built on it.  Shared by the CPU oracle (phaser_oracle.c) and
 * the FFTW-API shim (fftw_shim.c) that lets the reference's SOFT sources be
 * compiled here.  Written from the textbook definitions:
 *   DFT:     X[k] = sum_j x[j] exp(sign * 2 pi i jk / n)
 *   REDFT10: Y[k] = 2 sum_j x[j] cos(pi k (2j+1) / (2n))
 * TEST INFRASTRUCTURE ONLY.
 */
#ifndef ORACLE_FFT64_H_
#define ORACLE_FFT64_H_

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  double re, im;
} cplx;

static inline cplx cmul(cplx a, cplx b) {
  cplx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
  return r;
}

/* ------------------------------------------------------------------------ */
/* FFT: Stockham auto-sort, mixed radix, any length, FP64.                   */
/* Forward = exp(-2 pi i jk/n) (sign = -1), unnormalised.                    */
/* ------------------------------------------------------------------------ */

typedef struct {
  int n;
  int nf;
  int fac[40];
  cplx* w; /* w[t] = exp(-2 pi i t / n) */
} orc_fft_plan;

static inline void plan_init(orc_fft_plan* p, int n) {
  p->n = n;
  p->nf = 0;
  int m = n;
  while (m % 4 == 0) { p->fac[p->nf++] = 4; m /= 4; }
  while (m % 2 == 0) { p->fac[p->nf++] = 2; m /= 2; }
  for (int r = 3; m > 1; r += 2) {
    while (m % r == 0) { p->fac[p->nf++] = r; m /= r; }
  }
  p->w = (cplx*)malloc(sizeof(cplx) * (size_t)(n > 0 ? n : 1));
  for (int t = 0; t < n; ++t) {
    double a = -2.0 * M_PI * (double)t / (double)n;
    p->w[t].re = cos(a);
    p->w[t].im = sin(a);
  }
}

static inline void plan_free(orc_fft_plan* p) { free(p->w); p->w = NULL; }

/* exp(sign * 2 pi i t / n) from the table. */
static inline cplx tw(const orc_fft_plan* p, long t, int sign) {
  long n = p->n;
  t %= n;
  if (t < 0) t += n;
  cplx w = p->w[t];
  if (sign > 0) w.im = -w.im;
  return w;
}

/* In-place transform of x (length n) using scratch y (length n). */
static inline void fft_exec(const orc_fft_plan* p, cplx* x, cplx* y, int sign) {
  const int n = p->n;
  if (n <= 1) return;
  cplx* src = x;
  cplx* dst = y;
  int ns = 1;
  cplx v[64], o[64];
  for (int f = 0; f < p->nf; ++f) {
    const int R = p->fac[f];
    const int nr = n / R;
    for (int j = 0; j < nr; ++j) {
      const int k = j % ns;
      if (R <= 64) {
        for (int r = 0; r < R; ++r) {
          cplx a = src[j + r * nr];
          cplx t = tw(p, (long)r * k * (n / (ns * R)), sign);
          v[r] = cmul(a, t);
        }
        for (int s = 0; s < R; ++s) {
          cplx acc = {0.0, 0.0};
          for (int r = 0; r < R; ++r) {
            cplx t = tw(p, (long)((r * s) % R) * (n / R), sign);
            cplx m = cmul(v[r], t);
            acc.re += m.re;
            acc.im += m.im;
          }
          o[s] = acc;
        }
        const int idx = (j / ns) * ns * R + k;
        for (int s = 0; s < R; ++s) dst[idx + s * ns] = o[s];
      } else {
        /* large prime radix: direct sums without the small buffers */
        const int idx = (j / ns) * ns * R + k;
        for (int s = 0; s < R; ++s) {
          cplx acc = {0.0, 0.0};
          for (int r = 0; r < R; ++r) {
            cplx a = src[j + r * nr];
            cplx t = tw(p, (long)r * k * (n / (ns * R)), sign);
            cplx m = cmul(a, t);
            cplx t2 = tw(p, (long)((long)r * s % R) * (n / R), sign);
            m = cmul(m, t2);
            acc.re += m.re;
            acc.im += m.im;
          }
          dst[idx + s * ns] = acc;
        }
      }
    }
    cplx* tmp = src;
    src = dst;
    dst = tmp;
    ns *= R;
  }
  if (src != x) memcpy(x, src, sizeof(cplx) * (size_t)n);
}


/* REDFT10 of even length n via one complex FFT of length n. */
static inline void dct2_exec(const orc_fft_plan* p, const double* x, double* y,
                             cplx* v, cplx* scr) {
  const int n = p->n;
  if (n % 2 != 0) {
    for (int k = 0; k < n; ++k) {
      double s = 0.0;
      for (int j = 0; j < n; ++j) s += x[j] * cos(M_PI * k * (2.0 * j + 1.0) / (2.0 * n));
      y[k] = 2.0 * s;
    }
    return;
  }
  for (int j = 0; j < n / 2; ++j) {
    v[j].re = x[2 * j];
    v[j].im = 0.0;
    v[n - 1 - j].re = x[2 * j + 1];
    v[n - 1 - j].im = 0.0;
  }
  fft_exec(p, v, scr, -1);
  for (int k = 0; k < n; ++k) {
    const double a = -M_PI * (double)k / (2.0 * n);
    y[k] = 2.0 * (v[k].re * cos(a) - v[k].im * sin(a));
  }
}

#endif  /* ORACLE_FFT64_H_ */
