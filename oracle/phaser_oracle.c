/*
 * phaser_oracle.c -- FP64 CPU oracle of PHASER's correspondence-free
 * registration hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load this library, and only as the
 * checker.  The product (phaser_b200/) never links, loads or calls it.
 *
 * Every function restates, in plain C and double precision, the behaviour of
 * the reference function cited beside it (paths relative to the ethz-asl/phaser
 * tree).  Nothing here is copied from the reference: the spherical-harmonic and
 * SO(3) parts are written from the mathematics (Driscoll-Healy quadrature,
 * L2-normalised associated Legendre functions and Wigner-d functions by their
 * three-term recurrences), and are cross-checked in tests against the
 * reference's own SOFT sources compiled by oracle/Makefile.
 *
 * Conventions kept on purpose (reference quirks):
 *   - projection and grid use the float/double promotions of the reference;
 *   - nearest neighbour: float L2^2 accumulated as ((0+dx^2)+dy^2)+dz^2,
 *     lowest index wins ties (FLANN's tie order is not reproducible);
 *   - Laplace-pyramid fusion is positional on the FFT-shifted linear index,
 *     including the band-table rounding quirk of PyramidStruct vs expand();
 *   - the inverse SO(3) transform follows SOFT's real-data shortcut: only one
 *     member of each pair (m1,m2)/(-m1,-m2) is synthesised, the other is its
 *     complex conjugate;
 *   - voxel binning: float edges, histc binary search, -1 bins wrapped to
 *     uint32 and the `lin > N^3` guard (aliasing of out-of-range x / y);
 *   - translation width |lo|+|hi|+1.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "fft64.h"

/* Public 1-D FFT (used by tests to check the transform itself). */
void orc_fft1d(double* data_re_im, int n, int sign) {
  orc_fft_plan p;
  plan_init(&p, n);
  cplx* y = (cplx*)malloc(sizeof(cplx) * (size_t)n);
  fft_exec(&p, (cplx*)data_re_im, y, sign);
  free(y);
  plan_free(&p);
}

/* Full 3-D complex FFT over an n0 x n1 x n2 row-major array (n2 fastest). */
static void fft3d(cplx* a, int n0, int n1, int n2, int sign) {
  orc_fft_plan p0, p1, p2;
  plan_init(&p0, n0);
  plan_init(&p1, n1);
  plan_init(&p2, n2);
  int nmax = n0 > n1 ? n0 : n1;
  if (n2 > nmax) nmax = n2;
  /* axis 2 (contiguous) */
#pragma omp parallel
  {
    cplx* row = (cplx*)malloc(sizeof(cplx) * (size_t)nmax);
    cplx* scr = (cplx*)malloc(sizeof(cplx) * (size_t)nmax);
#pragma omp for
    for (long r = 0; r < (long)n0 * n1; ++r) {
      cplx* base = a + r * n2;
      memcpy(row, base, sizeof(cplx) * (size_t)n2);
      fft_exec(&p2, row, scr, sign);
      memcpy(base, row, sizeof(cplx) * (size_t)n2);
    }
#pragma omp for
    for (long r = 0; r < (long)n0 * n2; ++r) {
      long i0 = r / n2, i2 = r % n2;
      for (int i1 = 0; i1 < n1; ++i1) row[i1] = a[(i0 * n1 + i1) * n2 + i2];
      fft_exec(&p1, row, scr, sign);
      for (int i1 = 0; i1 < n1; ++i1) a[(i0 * n1 + i1) * n2 + i2] = row[i1];
    }
#pragma omp for
    for (long r = 0; r < (long)n1 * n2; ++r) {
      for (int i0 = 0; i0 < n0; ++i0) row[i0] = a[(long)i0 * n1 * n2 + r];
      fft_exec(&p0, row, scr, sign);
      for (int i0 = 0; i0 < n0; ++i0) a[(long)i0 * n1 * n2 + r] = row[i0];
    }
    free(row);
    free(scr);
  }
  plan_free(&p0);
  plan_free(&p1);
  plan_free(&p2);
}

/* ------------------------------------------------------------------------ */
/* Signal utils (phaser_common/src/common/signal-utils.cc:5-19,             */
/* phaser_common/include/phaser/common/signal-utils.h:30-47).              */
/* ------------------------------------------------------------------------ */

uint32_t orc_sub2ind(uint32_t i, uint32_t j, uint32_t k, uint32_t rows,
                     uint32_t cols) {
  return (i * cols + j) + (rows * cols * k);
}

void orc_ind2sub(uint32_t lin, uint32_t rows, uint32_t cols, uint32_t* xyz) {
  xyz[1] = lin % cols;
  const int upd = (int)(lin / cols);
  xyz[0] = (uint32_t)upd % rows;
  xyz[2] = (uint32_t)upd / rows;
}

/* std::rotate(first, first + s, last): out[i] = in[(i + s) mod n]. */
static void rotate_left(cplx* a, size_t n, size_t s) {
  if (n == 0) return;
  s %= n;
  if (s == 0) return;
  cplx* tmp = (cplx*)malloc(sizeof(cplx) * n);
  for (size_t i = 0; i < n; ++i) tmp[i] = a[(i + s) % n];
  memcpy(a, tmp, sizeof(cplx) * n);
  free(tmp);
}

void orc_fftshift(double* re_im, size_t n) {
  rotate_left((cplx*)re_im, n, (n % 2 == 0) ? (n >> 1) : (n >> 1) + 1);
}

void orc_ifftshift(double* re_im, size_t n) {
  rotate_left((cplx*)re_im, n, n >> 1);
}

/* ------------------------------------------------------------------------ */
/* Laplace pyramid (phaser_core/src/backend/fusion/pyramid-struct.cc:17-29, */
/* laplace-pyramid.cc:13-184).                                              */
/* ------------------------------------------------------------------------ */

void orc_pyramid_struct(uint32_t n, int levels, float div, uint32_t* lb,
                        uint32_t* ub, uint32_t* coeffs) {
  uint32_t cur = n;
  for (int l = 0; l < levels; ++l) {
    const float lower = (float)cur / div;
    const uint32_t upper = (uint32_t)roundf((float)cur - lower);
    lb[l] = (uint32_t)roundf(lower);
    ub[l] = upper;
    coeffs[l] = upper - lb[l];
    cur = coeffs[l];
  }
}

/* Literal level-by-level fusion: reduce -> max-energy per level -> mean of
 * the last low pass -> expand.  channels: C arrays of n complex (re,im). */
void orc_fuse_channels_literal(const double* channels, int C, uint32_t n,
                               int levels, float div, double* out) {
  uint32_t lb[16], ub[16], co[16];
  orc_pyramid_struct(n, levels, div, lb, ub, co);
  const cplx* ch = (const cplx*)channels;
  /* current low-pass views (pointers into copies) */
  cplx** low = (cplx**)malloc(sizeof(cplx*) * (size_t)C);
  cplx** fused = (cplx**)malloc(sizeof(cplx*) * (size_t)levels);
  uint32_t* fused_n = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)levels);
  cplx** owned = (cplx**)calloc((size_t)C * (size_t)(levels + 1), sizeof(cplx*));
  for (int c = 0; c < C; ++c) {
    owned[c] = (cplx*)malloc(sizeof(cplx) * (size_t)n);
    memcpy(owned[c], ch + (size_t)c * n, sizeof(cplx) * n);
    low[c] = owned[c];
  }
  for (int l = 0; l < levels; ++l) {
    const uint32_t n_low = co[l];
    const uint32_t n_lap = l > 0 ? co[l - 1] : n;
    cplx** lap = (cplx**)malloc(sizeof(cplx*) * (size_t)C);
    cplx** newlow = (cplx**)malloc(sizeof(cplx*) * (size_t)C);
    for (int c = 0; c < C; ++c) {
      newlow[c] = (cplx*)malloc(sizeof(cplx) * (size_t)(n_low ? n_low : 1));
      lap[c] = (cplx*)malloc(sizeof(cplx) * (size_t)(n_lap ? n_lap : 1));
      memcpy(lap[c], low[c], sizeof(cplx) * n_lap);
      for (uint32_t i = lb[l]; i < ub[l]; ++i) {
        const uint32_t k = i - lb[l];
        newlow[c][k] = low[c][i];
        lap[c][i].re = lap[c][i].re - newlow[c][k].re;
        lap[c][i].im = lap[c][i].im - newlow[c][k].im;
      }
    }
    fused[l] = (cplx*)malloc(sizeof(cplx) * (size_t)(n_lap ? n_lap : 1));
    fused_n[l] = n_lap;
    for (uint32_t i = 0; i < n_lap; ++i) {
      int best = 0;
      double be = -1.0;
      for (int c = 0; c < C; ++c) {
        const double e0 = sqrt(lap[c][i].re * lap[c][i].re + lap[c][i].im * lap[c][i].im);
        const double e = e0 * e0;
        if (c == 0 || e > be) {
          be = e;
          best = c;
        }
      }
      fused[l][i] = lap[best][i];
    }
    for (int c = 0; c < C; ++c) {
      free(lap[c]);
      owned[(size_t)(l + 1) * C + c] = newlow[c];
      low[c] = newlow[c];
    }
    free(lap);
    free(newlow);
  }
  /* mean of last low pass */
  const uint32_t n_last = co[levels - 1];
  cplx* recon = (cplx*)malloc(sizeof(cplx) * (size_t)(n_last ? n_last : 1));
  for (uint32_t i = 0; i < n_last; ++i) {
    double ar = 0.0, ai = 0.0;
    for (int c = 0; c < C; ++c) {
      ar += low[c][i].re;
      ai += low[c][i].im;
    }
    recon[i].re = ar / (double)C;
    recon[i].im = ai / (double)C;
  }
  for (int l = levels - 1; l >= 0; --l) {
    const uint32_t nc = fused_n[l];
    const uint32_t lo = (uint32_t)roundf((float)nc / div);
    const uint32_t up = nc - lo;
    for (uint32_t i = lo; i < up; ++i) fused[l][i] = recon[i - lo];
    free(recon);
    recon = fused[l];
  }
  memcpy(out, recon, sizeof(cplx) * n);
  free(recon);
  for (size_t i = 0; i < (size_t)C * (size_t)(levels + 1); ++i) free(owned[i]);
  free(owned);
  free(low);
  free(fused);
  free(fused_n);
}

/* Positional form of the same rule: 0 = max-energy channel, 1 = zero,
 * 2 = channel mean.  p is the index in the FFT-shifted array. */
int orc_fusion_rule(uint32_t p, uint32_t n, int levels, float div) {
  uint32_t lb[16], ub[16], co[16];
  orc_pyramid_struct(n, levels, div, lb, ub, co);
  uint32_t cur_n = n;
  for (int l = 0; l < levels; ++l) {
    const uint32_t elo = (uint32_t)roundf((float)cur_n / div);
    const uint32_t eup = cur_n - elo;
    if (p >= elo && p < eup) {
      p -= elo;
      cur_n = co[l];
      continue;
    }
    if (p >= lb[l] && p < ub[l]) return 1;
    return 0;
  }
  return 2;
}

/* Apply the positional rule to C channels at one position. */
static cplx fuse_at(const cplx* vals, int C, int rule) {
  cplx r = {0.0, 0.0};
  if (rule == 1) return r;
  if (rule == 2) {
    double ar = 0.0, ai = 0.0;
    for (int c = 0; c < C; ++c) {
      ar += vals[c].re;
      ai += vals[c].im;
    }
    r.re = ar / (double)C;
    r.im = ai / (double)C;
    return r;
  }
  int best = 0;
  double be = -1.0;
  for (int c = 0; c < C; ++c) {
    const double e0 = sqrt(vals[c].re * vals[c].re + vals[c].im * vals[c].im);
    const double e = e0 * e0;
    if (c == 0 || e > be) {
      be = e;
      best = c;
    }
  }
  return vals[best];
}

/* ------------------------------------------------------------------------ */
/* S^2 sampling (phaser_common/src/common/spherical-sampler.cc:29-64,       */
/* spherical-projection.cc:19-41, phaser_common/src/model/point-cloud.cc:   */
/* 66-72,93-157).                                                           */
/* ------------------------------------------------------------------------ */

void orc_dh_grid(int bw, float* xyz) {
  const int n = 2 * bw;
  for (int i = 0; i < n; ++i) {
    const float th = (float)((M_PI * (double)(2 * i + 1)) / (double)(4 * bw));
    for (int j = 0; j < n; ++j) {
      const float ph = (float)((2.0 * M_PI * (double)j) / (double)(2 * bw));
      const float dist = 1.0f;
      float* o = xyz + 3 * ((size_t)i * n + j);
      o[0] = dist * sinf(th) * cosf(ph);
      o[1] = dist * sinf(th) * sinf(ph);
      o[2] = dist * cosf(th);
    }
  }
}

void orc_project(const float* pts, size_t stride, size_t P, float* out_xyz,
                 double* range) {
  for (size_t i = 0; i < P; ++i) {
    const float x = pts[i * stride + 0];
    const float y = pts[i * stride + 1];
    const float z = pts[i * stride + 2];
    const float sxy = x * x + y * y;
    const double dist_xy = (double)sqrtf(sxy);
    const float zz = z * z;
    const double dist = sqrt(dist_xy * dist_xy + (double)zz);
    const float oz = (float)((double)z / dist);
    const double tx = (double)acosf(oz);
    const double ty = fmod((double)atan2f(y, x) + 2.0 * M_PI, 2.0 * M_PI);
    out_xyz[3 * i + 0] = (float)(sin(tx) * cos(ty));
    out_xyz[3 * i + 1] = (float)(sin(tx) * sin(ty));
    out_xyz[3 * i + 2] = oz;
    range[i] = dist;
  }
}

/* Exact float 1-NN (brute force).  Returns per query the index (or -1 when
 * rejected by max_sq_dist) and the float squared distance. */
void orc_nn(const float* q, size_t nq, const float* p, size_t np,
            float max_sq_dist, int32_t* idx, float* d2) {
#pragma omp parallel for schedule(dynamic, 64)
  for (long i = 0; i < (long)nq; ++i) {
    const float qx = q[3 * i], qy = q[3 * i + 1], qz = q[3 * i + 2];
    float best = INFINITY;
    int32_t bi = -1;
    for (size_t j = 0; j < np; ++j) {
      const float dx = qx - p[3 * j];
      const float dy = qy - p[3 * j + 1];
      const float dz = qz - p[3 * j + 2];
      float r = 0.0f;
      r += dx * dx;
      r += dy * dy;
      r += dz * dz;
      if (r < best) {
        best = r;
        bi = (int32_t)j;
      }
    }
    d2[i] = best;
    idx[i] = (bi >= 0 && !(best > max_sq_dist)) ? bi : -1;
  }
}

/* Sample a cloud on the 2B x 2B DH grid.  Output channel order
 * {range, intensity, reflectivity, ambient} (spherical-combined-worker.cc:
 * 19-59); out has 4 * 4B^2 doubles, [channel][theta][phi]. */
void orc_sample_cloud(const float* xyzi, size_t P, const float* refl,
                      const float* amb, int bw, float max_sq_dist, double* out,
                      int32_t* nn_idx_out) {
  const size_t nq = (size_t)4 * bw * bw;
  float* grid = (float*)malloc(sizeof(float) * 3 * nq);
  orc_dh_grid(bw, grid);
  float* proj = (float*)malloc(sizeof(float) * 3 * (P ? P : 1));
  double* rng = (double*)malloc(sizeof(double) * (P ? P : 1));
  orc_project(xyzi, 4, P, proj, rng);
  int32_t* idx = (int32_t*)malloc(sizeof(int32_t) * nq);
  float* d2 = (float*)malloc(sizeof(float) * nq);
  orc_nn(grid, nq, proj, P, max_sq_dist, idx, d2);
  for (size_t i = 0; i < nq; ++i) {
    const int32_t j = idx[i];
    double r = 0.0, it = 0.0, rf = 0.0, am = 0.0;
    if (j >= 0) {
      r = rng[j];
      it = (double)xyzi[4 * (size_t)j + 3];
      rf = refl ? (double)refl[j] : 0.0;
      am = amb ? (double)amb[j] : 0.0;
    }
    out[0 * nq + i] = r;
    out[1 * nq + i] = it;
    out[2 * nq + i] = rf;
    out[3 * nq + i] = am;
    if (nn_idx_out) nn_idx_out[i] = j;
  }
  free(grid);
  free(proj);
  free(rng);
  free(idx);
  free(d2);
}

/* ------------------------------------------------------------------------ */
/* Forward SHT (behaviour of SOFT FST_semi_memo with cutoff = bw on real    */
/* data, phaser_core/lib/SOFT/s2_semi_memo.c:123-367): the semi-naive       */
/* algorithm evaluates exactly the Driscoll-Healy quadrature sum, so the    */
/* oracle computes that sum directly:                                       */
/*   F_m(theta_k) = sqrt(2 pi)/(2B) sum_j f(theta_k, phi_j) e^{-i m phi_j}  */
/*   fhat(l,m)    = sum_k w_k Pbar_l^m(cos theta_k) F_m(theta_k)            */
/* with Pbar L2-normalised on [-1,1] including the Condon-Shortley phase.  */
/* Output in the seanindex order of s2_primitive.c:300-311.                 */
/* ------------------------------------------------------------------------ */

int orc_seanindex(int m, int l, int bw) {
  const int L = bw - 1;
  if (m >= 0) return m * (L + 1) - ((m * (m - 1)) / 2) + (l - m);
  return ((L * (L + 3)) / 2) + 1 + ((L + m) * (L + m + 1) / 2) + (l - abs(m));
}

/* Driscoll-Healy quadrature weights for 2B Chebyshev-type nodes. */
void orc_dh_weights(int bw, double* w) {
  for (int k = 0; k < 2 * bw; ++k) {
    const double th = M_PI * (2.0 * k + 1.0) / (4.0 * bw);
    double s = 0.0;
    for (int i = 0; i < bw; ++i) s += sin((2.0 * i + 1.0) * th) / (2.0 * i + 1.0);
    w[k] = (2.0 / (double)bw) * sin(th) * s;
  }
}

/* Pbar_l^m(x) for l = m..bw-1 at one x (FP64 recurrence). */
static void legendre_column(int m, int bw, double x, double sin_t, double* out) {
  /* seed Pbar_m^m = (-1)^m sqrt((2m+1)/2 * (2m)!/(4^m (m!)^2)) sin^m */
  double c = sqrt((2.0 * m + 1.0) / 2.0);
  for (int i = 1; i <= m; ++i) c *= sqrt((2.0 * i - 1.0) / (2.0 * i));
  double pmm = c * pow(sin_t, (double)m);
  if (m & 1) pmm = -pmm;
  out[0] = pmm;
  if (m + 1 >= bw) return;
  double p_prev = 0.0, p_cur = pmm;
  for (int l = m; l + 1 < bw; ++l) {
    const double a = sqrt((2.0 * l + 1.0) * (2.0 * l + 3.0) /
                          ((double)(l + 1 - m) * (double)(l + 1 + m)));
    const double b = (l > m) ? sqrt((2.0 * l + 3.0) * (double)(l - m) * (double)(l + m) /
                                    ((2.0 * l - 1.0) * (double)(l + 1 - m) * (double)(l + 1 + m)))
                             : 0.0;
    const double p_next = a * x * p_cur - b * p_prev;
    out[l + 1 - m] = p_next;
    p_prev = p_cur;
    p_cur = p_next;
  }
}

/* Forward SHT of one real 2B x 2B signal [theta][phi].  coef_re/im: B^2. */
void orc_sht(const double* sig, int bw, double* coef_re, double* coef_im) {
  const int n = 2 * bw;
  double* w = (double*)malloc(sizeof(double) * n);
  orc_dh_weights(bw, w);
  cplx* Fm = (cplx*)malloc(sizeof(cplx) * (size_t)bw * n); /* [m][k] */
  const double scale = sqrt(2.0 * M_PI) / (double)n;
  double* ct = (double*)malloc(sizeof(double) * n);
  double* st = (double*)malloc(sizeof(double) * n);
  for (int t = 0; t < n; ++t) {
    const double a = -2.0 * M_PI * (double)t / (double)n;
    ct[t] = cos(a);
    st[t] = sin(a);
  }
  for (int k = 0; k < n; ++k) {
    for (int m = 0; m < bw; ++m) {
      double ar = 0.0, ai = 0.0;
      for (int j = 0; j < n; ++j) {
        const int t = (int)((long)j * m % n);
        ar += sig[(size_t)k * n + j] * ct[t];
        ai += sig[(size_t)k * n + j] * st[t];
      }
      Fm[(size_t)m * n + k].re = ar * scale;
      Fm[(size_t)m * n + k].im = ai * scale;
    }
  }
  free(ct);
  free(st);
  double* col = (double*)malloc(sizeof(double) * bw);
  double* acc_re = (double*)calloc((size_t)bw * bw, sizeof(double));
  double* acc_im = (double*)calloc((size_t)bw * bw, sizeof(double));
  for (int m = 0; m < bw; ++m) {
    for (int k = 0; k < n; ++k) {
      const double th = M_PI * (2.0 * k + 1.0) / (4.0 * bw);
      legendre_column(m, bw, cos(th), sin(th), col);
      for (int l = m; l < bw; ++l) {
        const double f = w[k] * col[l - m];
        acc_re[(size_t)m * bw + l] += f * Fm[(size_t)m * n + k].re;
        acc_im[(size_t)m * bw + l] += f * Fm[(size_t)m * n + k].im;
      }
    }
  }
  for (int m = 0; m < bw; ++m) {
    for (int l = m; l < bw; ++l) {
      const int ip = orc_seanindex(m, l, bw);
      coef_re[ip] = acc_re[(size_t)m * bw + l];
      coef_im[ip] = acc_im[(size_t)m * bw + l];
      if (m > 0) {
        const int in = orc_seanindex(-m, l, bw);
        const double sgn = (m & 1) ? -1.0 : 1.0;
        coef_re[in] = sgn * coef_re[ip];
        coef_im[in] = -sgn * coef_im[ip];
      }
    }
  }
  free(w);
  free(Fm);
  free(col);
  free(acc_re);
  free(acc_im);
}

/* ------------------------------------------------------------------------ */
/* Wigner-d, L2-normalised in beta (int_0^pi d^2 sin = 1), standard sign     */
/* convention d^j_{m1 m2}(beta) = <j m1| exp(-i beta J_y) |j m2>.          */
/* Seed at j = max(|m1|,|m2|) from the closed form, then the three-term     */
/* recurrence in j.  Same functions as SOFT makeWigner.c:180-210,324-387.   */
/* ------------------------------------------------------------------------ */

static double wig_seed(int m1, int m2, double beta) {
  const int a1 = abs(m1), a2 = abs(m2);
  const int j = a1 > a2 ? a1 : a2;
  const int mn = a1 < a2 ? a1 : a2;
  int cp, sp;
  double sgn = 1.0;
  if (j == a1) {
    if (m1 >= 0) {
      cp = j + m2;
      sp = j - m2;
      if ((j - m2) & 1) sgn = -1.0;
    } else {
      cp = j - m2;
      sp = j + m2;
    }
  } else if (m2 >= 0) {
    cp = j + m1;
    sp = j - m1;
  } else {
    cp = j - m1;
    sp = j + m1;
    if ((j + m1) & 1) sgn = -1.0;
  }
  /* sqrt((2j+1)/2 * C(2j, j-mn)) */
  double nf = 1.0;
  for (int i = 0; i < j - mn; ++i) nf *= sqrt((2.0 * j - i) / (i + 1.0));
  nf *= sqrt((2.0 * j + 1.0) / 2.0);
  return sgn * nf * pow(sin(0.5 * beta), (double)sp) * pow(cos(0.5 * beta), (double)cp);
}

/* Recurrence coefficients for orders (m1,m2), l = j0 .. bw-2:
 *   d^{l+1} = fa[l] d^{l-1} + fb[l] (cos beta + sh[l]) d^l. */
static void wig_coeffs(int m1, int m2, int bw, double* fa, double* fb, double* sh) {
  const int a1 = abs(m1), a2 = abs(m2);
  const int j0 = a1 > a2 ? a1 : a2;
  const double dm1 = m1, dm2 = m2;
  for (int l = j0; l + 1 < bw; ++l) {
    const double dl = l;
    const double tnext = sqrt(((dl + 1) * (dl + 1) - dm1 * dm1) * ((dl + 1) * (dl + 1) - dm2 * dm2));
    fb[l] = sqrt((2 * dl + 3) / (2 * dl + 1)) * (dl + 1) * (2 * dl + 1) / tnext;
    sh[l] = (l == 0) ? 0.0 : -dm1 * dm2 / (dl * (dl + 1));
    fa[l] = 0.0;
    if (l > 0) {
      const double tcur = sqrt((dl * dl - dm1 * dm1) * (dl * dl - dm2 * dm2));
      fa[l] = -sqrt((2 * dl + 3) / (2 * dl - 1)) * (dl + 1) / dl * tcur / tnext;
    }
  }
}

static void wig_run(int m1, int m2, int bw, double beta, const double* fa,
                    const double* fb, const double* sh, double* out) {
  const int a1 = abs(m1), a2 = abs(m2);
  const int j0 = a1 > a2 ? a1 : a2;
  if (j0 >= bw) return;
  double dprev = 0.0;
  double dcur = wig_seed(m1, m2, beta);
  out[0] = dcur;
  const double cb = cos(beta);
  for (int l = j0; l + 1 < bw; ++l) {
    const double dnext = fa[l] * dprev + fb[l] * (cb + sh[l]) * dcur;
    out[l + 1 - j0] = dnext;
    dprev = dcur;
    dcur = dnext;
  }
}

/* d^l_{m1 m2}(beta) for l = j0 .. bw-1 into out[l - j0]. */
void orc_wigner_column(int m1, int m2, int bw, double beta, double* out) {
  double* fa = (double*)malloc(sizeof(double) * (bw + 1));
  double* fb = (double*)malloc(sizeof(double) * (bw + 1));
  double* sh = (double*)malloc(sizeof(double) * (bw + 1));
  wig_coeffs(m1, m2, bw, fa, fb, sh);
  wig_run(m1, m2, bw, beta, fa, fb, sh, out);
  free(fa);
  free(fb);
  free(sh);
}

/* so3 coefficient product (so3_correlate_fftw.c:102-161): for l < bw_in,
 *   c(l,m1,m2) = 2 pi sqrt(2/(2l+1)) fhat(l,-m1) (-1)^(m1+m2) conj(hhat(l,-m2)).
 * Membership of the synthesised half (soft_fftw.c:1036-1914 with flag=1). */
static int in_half(int a, int b) {
  if (a > 0) return !(b == -a);
  if (a == 0) return b >= 0;
  return b == -a; /* (-m, m), m >= 1 */
}

/* Inverse SO(3) correlation volume, complex [beta][alpha][gamma] with gamma
 * fastest, (2 bw_out)^3 entries, from S^2 coefficients (seanindex, bw_in). */
void orc_so3_correlate(int bw_in, int bw_out, const double* f_re,
                       const double* f_im, const double* h_re,
                       const double* h_im, double* out_re_im) {
  const int n = 2 * bw_out;
  const size_t n2 = (size_t)n * n;
  cplx* vol = (cplx*)out_re_im;
  memset(vol, 0, sizeof(cplx) * n2 * n);
  /* S[beta][a_idx][b_idx] */
#pragma omp parallel
  {
    double* d = (double*)malloc(sizeof(double) * (bw_in > 0 ? bw_in : 1));
    double* fa = (double*)malloc(sizeof(double) * (bw_in + 1));
    double* fb = (double*)malloc(sizeof(double) * (bw_in + 1));
    double* sh = (double*)malloc(sizeof(double) * (bw_in + 1));
#pragma omp for schedule(dynamic, 1)
    for (int ai = 0; ai < 2 * bw_in - 1; ++ai) {
      const int a = ai - (bw_in - 1);
      for (int b = -(bw_in - 1); b <= bw_in - 1; ++b) {
        if (!in_half(a, b)) continue;
        const int j0 = abs(a) > abs(b) ? abs(a) : abs(b);
        if (j0 >= bw_in) continue;
        const int aidx = (a + n) % n, bidx = (b + n) % n;
        const int caidx = (-a + n) % n, cbidx = (-b + n) % n;
        wig_coeffs(a, b, bw_in, fa, fb, sh);
        for (int k = 0; k < n; ++k) {
          const double beta = M_PI * (2.0 * k + 1.0) / (4.0 * bw_out);
          wig_run(a, b, bw_in, beta, fa, fb, sh, d);
          double sr = 0.0, si = 0.0;
          for (int l = j0; l < bw_in; ++l) {
            const int i1 = orc_seanindex(-a, l, bw_in);
            const int i2 = orc_seanindex(-b, l, bw_in);
            const double fr = f_re[i1], fi = f_im[i1];
            const double sg = ((a + b) & 1) ? -1.0 : 1.0;
            const double pr = sg * h_re[i2], pi = sg * -h_im[i2];
            const double wn = 2.0 * M_PI * sqrt(2.0 / (2.0 * l + 1.0));
            const double cr = wn * (fr * pr - fi * pi);
            const double ci = wn * (fr * pi + fi * pr);
            sr += cr * d[l - j0];
            si += ci * d[l - j0];
          }
          cplx* s = &vol[(size_t)k * n2 + (size_t)aidx * n + bidx];
          s->re = sr;
          s->im = si;
          if (!(a == 0 && b == 0)) {
            cplx* c = &vol[(size_t)k * n2 + (size_t)caidx * n + cbidx];
            c->re = sr;
            c->im = -si;
          }
        }
      }
    }
    free(d);
    free(fa);
    free(fb);
    free(sh);
  }
  /* 2-D forward DFT over (a, b) -> (alpha, gamma) per beta, scaled. */
  orc_fft_plan p;
  plan_init(&p, n);
  const double sc = (1.0 / (double)n) * ((double)bw_out / M_PI);
#pragma omp parallel
  {
    cplx* row = (cplx*)malloc(sizeof(cplx) * n);
    cplx* scr = (cplx*)malloc(sizeof(cplx) * n);
#pragma omp for
    for (int k = 0; k < n; ++k) {
      cplx* sl = vol + (size_t)k * n2;
      for (int ai = 0; ai < n; ++ai) {
        memcpy(row, sl + (size_t)ai * n, sizeof(cplx) * n);
        fft_exec(&p, row, scr, -1);
        memcpy(sl + (size_t)ai * n, row, sizeof(cplx) * n);
      }
      for (int bi = 0; bi < n; ++bi) {
        for (int ai = 0; ai < n; ++ai) row[ai] = sl[(size_t)ai * n + bi];
        fft_exec(&p, row, scr, -1);
        for (int ai = 0; ai < n; ++ai) {
          sl[(size_t)ai * n + bi].re = row[ai].re * sc;
          sl[(size_t)ai * n + bi].im = row[ai].im * sc;
        }
      }
    }
    free(row);
    free(scr);
  }
  plan_free(&p);
}

/* SphericalCorrelationLaplace::correlateSampledSignals
 * (spherical-correlation-laplace.cc:14-40): C >= 2 channels per side, each a
 * 4B^2 signal; output corr = |z|^2 over (2 bw_out)^3.  mode 1 = the single-
 * signal SphericalCorrelation path (C = 1, no fusion). */
void orc_spherical_correlation(int bw, int bw_out, int C, const double* f,
                               const double* g, int levels, double* corr,
                               double* fused_f_re_im, double* fused_g_re_im) {
  const size_t nc = (size_t)bw * bw;
  const size_t ns = (size_t)4 * bw * bw;
  double* fr = (double*)malloc(sizeof(double) * nc * C);
  double* fi = (double*)malloc(sizeof(double) * nc * C);
  double* gr = (double*)malloc(sizeof(double) * nc * C);
  double* gi = (double*)malloc(sizeof(double) * nc * C);
  for (int c = 0; c < C; ++c) {
    orc_sht(f + ns * c, bw, fr + nc * c, fi + nc * c);
    orc_sht(g + ns * c, bw, gr + nc * c, gi + nc * c);
  }
  double* Ff_re = (double*)malloc(sizeof(double) * nc);
  double* Ff_im = (double*)malloc(sizeof(double) * nc);
  double* Gf_re = (double*)malloc(sizeof(double) * nc);
  double* Gf_im = (double*)malloc(sizeof(double) * nc);
  if (C == 1) {
    memcpy(Ff_re, fr, sizeof(double) * nc);
    memcpy(Ff_im, fi, sizeof(double) * nc);
    memcpy(Gf_re, gr, sizeof(double) * nc);
    memcpy(Gf_im, gi, sizeof(double) * nc);
  } else {
    cplx* vf = (cplx*)malloc(sizeof(cplx) * C);
    cplx* vg = (cplx*)malloc(sizeof(cplx) * C);
    for (size_t k = 0; k < nc; ++k) {
      const uint32_t p = (uint32_t)((k + (nc >> 1)) % nc);
      const int rule = orc_fusion_rule(p, (uint32_t)nc, levels, 4.0f);
      for (int c = 0; c < C; ++c) {
        vf[c].re = fr[nc * c + k];
        vf[c].im = fi[nc * c + k];
        vg[c].re = gr[nc * c + k];
        vg[c].im = gi[nc * c + k];
      }
      const cplx a = fuse_at(vf, C, rule);
      const cplx b = fuse_at(vg, C, rule);
      Ff_re[k] = a.re;
      Ff_im[k] = a.im;
      Gf_re[k] = b.re;
      Gf_im[k] = b.im;
    }
    free(vf);
    free(vg);
  }
  if (fused_f_re_im) {
    for (size_t k = 0; k < nc; ++k) {
      fused_f_re_im[2 * k] = Ff_re[k];
      fused_f_re_im[2 * k + 1] = Ff_im[k];
      fused_g_re_im[2 * k] = Gf_re[k];
      fused_g_re_im[2 * k + 1] = Gf_im[k];
    }
  }
  /* corr NULL: the fused spectra alone */
  if (corr) {
    const int n = 2 * bw_out;
    const size_t nv = (size_t)n * n * n;
    double* vol = (double*)malloc(sizeof(double) * 2 * nv);
    orc_so3_correlate(bw, bw_out, Ff_re, Ff_im, Gf_re, Gf_im, vol);
    for (size_t i = 0; i < nv; ++i)
      corr[i] = vol[2 * i] * vol[2 * i] + vol[2 * i + 1] * vol[2 * i + 1];
    free(vol);
  }
  free(fr);
  free(fi);
  free(gr);
  free(gi);
  free(Ff_re);
  free(Ff_im);
  free(Gf_re);
  free(Gf_im);
}

/* |z|^2 of the correlation at the listed beta indices only (the same
 * coefficient product, Wigner-d recurrence and angle transforms as
 * orc_so3_correlate, restricted to nk slices: [nk][alpha][gamma]), from the
 * fused spectra of orc_spherical_correlation.  For bandwidths whose full
 * FP64 volume is too large to evaluate. */
void orc_so3_correlate_slices(int bw_in, int bw_out, const double* f_re, const double* f_im, const double* h_re,
                              const double* h_im, int nk, const int* ks, double* out) {
  const int n = 2 * bw_out;
  const size_t n2 = (size_t)n * n;
  cplx* sl_all = (cplx*)calloc((size_t)nk * n2, sizeof(cplx));
#pragma omp parallel
  {
    double* d = (double*)malloc(sizeof(double) * (bw_in > 0 ? bw_in : 1));
    double* fa = (double*)malloc(sizeof(double) * (bw_in + 1));
    double* fb = (double*)malloc(sizeof(double) * (bw_in + 1));
    double* sh = (double*)malloc(sizeof(double) * (bw_in + 1));
#pragma omp for schedule(dynamic, 1)
    for (int ai = 0; ai < 2 * bw_in - 1; ++ai) {
      const int a = ai - (bw_in - 1);
      for (int b = -(bw_in - 1); b <= bw_in - 1; ++b) {
        if (!in_half(a, b)) continue;
        const int j0 = abs(a) > abs(b) ? abs(a) : abs(b);
        if (j0 >= bw_in) continue;
        const int aidx = (a + n) % n, bidx = (b + n) % n;
        const int caidx = (-a + n) % n, cbidx = (-b + n) % n;
        wig_coeffs(a, b, bw_in, fa, fb, sh);
        for (int s = 0; s < nk; ++s) {
          const int k = ks[s];
          const double beta = M_PI * (2.0 * k + 1.0) / (4.0 * bw_out);
          wig_run(a, b, bw_in, beta, fa, fb, sh, d);
          double sr = 0.0, si = 0.0;
          for (int l = j0; l < bw_in; ++l) {
            const int i1 = orc_seanindex(-a, l, bw_in);
            const int i2 = orc_seanindex(-b, l, bw_in);
            const double fr = f_re[i1], fi = f_im[i1];
            const double sg = ((a + b) & 1) ? -1.0 : 1.0;
            const double pr = sg * h_re[i2], pi = sg * -h_im[i2];
            const double wn = 2.0 * M_PI * sqrt(2.0 / (2.0 * l + 1.0));
            sr += wn * (fr * pr - fi * pi) * d[l - j0];
            si += wn * (fr * pi + fi * pr) * d[l - j0];
          }
          cplx* sl = sl_all + (size_t)s * n2;
          sl[(size_t)aidx * n + bidx].re = sr;
          sl[(size_t)aidx * n + bidx].im = si;
          if (!(a == 0 && b == 0)) {
            sl[(size_t)caidx * n + cbidx].re = sr;
            sl[(size_t)caidx * n + cbidx].im = -si;
          }
        }
      }
    }
    free(d);
    free(fa);
    free(fb);
    free(sh);
  }
  orc_fft_plan p;
  plan_init(&p, n);
  const double sc = (1.0 / (double)n) * ((double)bw_out / M_PI);
#pragma omp parallel
  {
    cplx* row = (cplx*)malloc(sizeof(cplx) * n);
    cplx* scr = (cplx*)malloc(sizeof(cplx) * n);
#pragma omp for
    for (int s = 0; s < nk; ++s) {
      cplx* sl = sl_all + (size_t)s * n2;
      for (int ai = 0; ai < n; ++ai) {
        memcpy(row, sl + (size_t)ai * n, sizeof(cplx) * n);
        fft_exec(&p, row, scr, -1);
        memcpy(sl + (size_t)ai * n, row, sizeof(cplx) * n);
      }
      for (int bi = 0; bi < n; ++bi) {
        for (int ai = 0; ai < n; ++ai) row[ai] = sl[(size_t)ai * n + bi];
        fft_exec(&p, row, scr, -1);
        for (int ai = 0; ai < n; ++ai) {
          const double re = row[ai].re * sc, im = row[ai].im * sc;
          out[(size_t)s * n2 + (size_t)ai * n + bi] = re * re + im * im;
        }
      }
    }
    free(row);
    free(scr);
  }
  plan_free(&p);
  free(sl_all);
}

/* Raw signed volume (real part) for error measurements. */
void orc_spherical_volume(int bw, int bw_out, int C, const double* f,
                          const double* g, int levels, double* vol_re_im) {
  const size_t nc = (size_t)bw * bw;
  double* ff = (double*)malloc(sizeof(double) * 2 * nc);
  double* gg = (double*)malloc(sizeof(double) * 2 * nc);
  const int n = 2 * bw_out;
  double* corr = (double*)malloc(sizeof(double) * (size_t)n * n * n);
  orc_spherical_correlation(bw, bw_out, C, f, g, levels, corr, ff, gg);
  double* fr = (double*)malloc(sizeof(double) * nc);
  double* fi = (double*)malloc(sizeof(double) * nc);
  double* gr = (double*)malloc(sizeof(double) * nc);
  double* gi = (double*)malloc(sizeof(double) * nc);
  for (size_t k = 0; k < nc; ++k) {
    fr[k] = ff[2 * k];
    fi[k] = ff[2 * k + 1];
    gr[k] = gg[2 * k];
    gi[k] = gg[2 * k + 1];
  }
  orc_so3_correlate(bw, bw_out, fr, fi, gr, gi, vol_re_im);
  free(ff);
  free(gg);
  free(corr);
  free(fr);
  free(fi);
  free(gr);
  free(gi);
}

/* First-occurrence argmax (z-score-eval.cc:46,56). */
uint64_t orc_argmax(const double* v, uint64_t n) {
  uint64_t b = 0;
  for (uint64_t i = 1; i < n; ++i)
    if (v[i] > v[b]) b = i;
  return b;
}

/* ------------------------------------------------------------------------ */
/* Rotation bin -> pose (phaser_common/src/common/rotation-utils.cc:17-24,  */
/* 86-143, 190-208; bingham-peak-based-eval.cc with 0 neighbours: the mode  */
/* of a one-sample Bingham fit is +-q of the bin).                          */
/* ------------------------------------------------------------------------ */

void orc_bin_to_zyz(uint32_t loc, uint32_t bw, double* zyz) {
  const int32_t ii = (int32_t)floor(loc / (4. * bw * bw));
  int32_t tmp = (int32_t)(loc - (ii * 4. * bw * bw));
  const int32_t jj = (int32_t)floor(tmp / (2. * bw));
  const int32_t kk = (int32_t)loc - (ii * 4 * (int32_t)bw * (int32_t)bw) - jj * (2 * (int32_t)bw);
  const double b = (double)bw;
  zyz[0] = M_PI * jj / b;
  zyz[1] = M_PI * (2 * ii + 1) / (4. * bw);
  zyz[2] = M_PI * kk / b;
}

static void quat_mul(const double* a, const double* b, double* r) {
  /* (w, x, y, z) Hamilton product */
  r[0] = a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3];
  r[1] = a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2];
  r[2] = a[0] * b[2] - a[1] * b[3] + a[2] * b[0] + a[3] * b[1];
  r[3] = a[0] * b[3] + a[1] * b[2] - a[2] * b[1] + a[3] * b[0];
}

void orc_zyz_to_quat(const double* zyz, double* q) {
  const double qa[4] = {cos(zyz[0] / 2), 0, 0, sin(zyz[0] / 2)};
  const double qb[4] = {cos(zyz[1] / 2), 0, sin(zyz[1] / 2), 0};
  const double qc[4] = {cos(zyz[2] / 2), 0, 0, sin(zyz[2] / 2)};
  double t[4];
  quat_mul(qa, qb, t);
  quat_mul(t, qc, q);
}

void orc_quat_to_xyz(const double* q, double* xyz) {
  const double qw = q[0], qx = q[1], qy = q[2], qz = q[3];
  const double r11 = -2 * (qy * qz - qw * qx);
  const double r12 = qw * qw - qx * qx - qy * qy + qz * qz;
  const double r21 = 2 * (qx * qz + qw * qy);
  const double r31 = -2 * (qx * qy - qw * qz);
  const double r32 = qw * qw + qx * qx - qy * qy - qz * qz;
  xyz[2] = -atan2(r31, r32);
  xyz[1] = asin(r21);
  xyz[0] = atan2(r11, r12);
}

/* Rx(a) * Ry(b) * Rz(c) as float 3x4 (rows), createTransformationAround*
 * (phaser_common/src/common/rotation-utils.cc:109-143).  std::cos(float) and
 * std::sin(float) are taken as their correctly rounded values (evaluated in
 * double, rounded once): the reference's libm is not pinned, and glibc 2.39's
 * cosf / sinf differ from the correctly rounded value on ~1.3% of inputs. */
static float cr_cosf(float x) { return (float)cos((double)x); }
static float cr_sinf(float x) { return (float)sin((double)x); }

void orc_rotation_xyz(float a, float b, float c, float* T) {
  const float ca = cr_cosf(a), sa = cr_sinf(a);
  const float cb = cr_cosf(b), sb = cr_sinf(b);
  const float cc = cr_cosf(c), sc = cr_sinf(c);
  float X[3][3] = {{1, 0, 0}, {0, ca, -sa}, {0, sa, ca}};
  float Y[3][3] = {{cb, 0, sb}, {0, 1, 0}, {-sb, 0, cb}};
  float Z[3][3] = {{cc, sc, 0}, {-sc, cc, 0}, {0, 0, 1}};
  float XY[3][3], R[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      float s = 0.0f;
      for (int k = 0; k < 3; ++k) s += X[i][k] * Y[k][j];
      XY[i][j] = s;
    }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      float s = 0.0f;
      for (int k = 0; k < 3; ++k) s += XY[i][k] * Z[k][j];
      R[i][j] = s;
    }
  for (int i = 0; i < 3; ++i) {
    T[4 * i + 0] = R[i][0];
    T[4 * i + 1] = R[i][1];
    T[4 * i + 2] = R[i][2];
    T[4 * i + 3] = 0.0f;
  }
}

/* PCL 1.8 transformPointCloud order: ((T0 x + T1 y) + T2 z) + T3, float. */
void orc_transform(float* xyzi, size_t P, const float* T) {
  for (size_t i = 0; i < P; ++i) {
    const float x = xyzi[4 * i], y = xyzi[4 * i + 1], z = xyzi[4 * i + 2];
    float o[3];
    for (int r = 0; r < 3; ++r) {
      float s = T[4 * r + 0] * x;
      s = s + T[4 * r + 1] * y;
      s = s + T[4 * r + 2] * z;
      s = s + T[4 * r + 3];
      o[r] = s;
    }
    xyzi[4 * i] = o[0];
    xyzi[4 * i + 1] = o[1];
    xyzi[4 * i + 2] = o[2];
  }
}

/* ------------------------------------------------------------------------ */
/* Voxeliser (phaser_core/src/backend/alignment/phase-aligner.cc:27-30,     */
/* 71-131; phaser_core/include/igl/histc.cpp:34-73).                        */
/* ------------------------------------------------------------------------ */

/* Eigen::VectorXf::LinSpaced(N, lo, hi) of Eigen >= 3.3 (the eigen_catkin
 * version phaser builds against; Eigen's published linspaced_op for floats):
 * step = (hi - lo) / (N - 1) in float; when |hi| < |lo| the entries count
 * down from the high end, e[0] = lo, e[i] = hi - (N - 1 - i) step, otherwise
 * up from the low end, e[i] = lo + i step, e[N - 1] = hi. */
void orc_edges(int N, int lo, int hi, float* e) {
  const float flo = (float)lo, fhi = (float)hi;
  const float step = (N == 1) ? 0.0f : (fhi - flo) / (float)(N - 1);
  const int flip = fabsf(fhi) < fabsf(flo);
  for (int i = 0; i < N; ++i) {
    if (flip)
      e[i] = (i == 0) ? flo : (fhi - (float)(N - 1 - i) * step);
    else
      e[i] = (i == N - 1) ? fhi : (flo + (float)i * step);
  }
}

static int32_t histc1(float xf, const float* E, int N) {
  const double x = (double)xf;
  if (x < (double)E[0] || x > (double)E[N - 1]) return -1;
  size_t l = 0, h = (size_t)N - 1, k = l;
  while ((h - l) > 1) {
    k = (h + l) / 2;
    if (x < (double)E[k])
      h = k;
    else
      l = k;
  }
  if (x == (double)E[h])
    k = h;
  else
    k = l;
  return (int32_t)k;
}

/* Per-point linear voxel index as the reference computes it (uint32 wrap),
 * or 0xFFFFFFFF when the `lin > N^3` guard skips the point. */
void orc_voxel_index(const float* xyzi, size_t P, int N, int lo, int hi,
                     uint32_t* lin_out) {
  float* E = (float*)malloc(sizeof(float) * N);
  orc_edges(N, lo, hi, E);
  const uint32_t nf = (uint32_t)N * (uint32_t)N * (uint32_t)N;
  for (size_t i = 0; i < P; ++i) {
    const uint32_t bx = (uint32_t)histc1(xyzi[4 * i], E, N);
    const uint32_t by = (uint32_t)histc1(xyzi[4 * i + 1], E, N);
    const uint32_t bz = (uint32_t)histc1(xyzi[4 * i + 2], E, N);
    const uint32_t lin = orc_sub2ind(bx, by, bz, (uint32_t)N, (uint32_t)N);
    lin_out[i] = (lin > nf || lin == nf) ? 0xFFFFFFFFu : lin;
  }
  free(E);
}

/* discretizePointcloud: out has 4 * N^3 doubles in the channel order
 * {intensity, range, reflectivity, ambient}; range = sqrtf(x^2+y^2+z^2). */
void orc_discretize(const float* xyzi, size_t P, const float* refl,
                    const float* amb, int N, int lo, int hi, double* out) {
  const size_t nv = (size_t)N * N * N;
  uint32_t* lin = (uint32_t*)malloc(sizeof(uint32_t) * (P ? P : 1));
  orc_voxel_index(xyzi, P, N, lo, hi, lin);
  double* hist = (double*)calloc(nv, sizeof(double));
  memset(out, 0, sizeof(double) * 4 * nv);
  for (size_t i = 0; i < P; ++i) {
    const uint32_t v = lin[i];
    if (v == 0xFFFFFFFFu) continue;
    const float x = xyzi[4 * i], y = xyzi[4 * i + 1], z = xyzi[4 * i + 2];
    out[0 * nv + v] = out[0 * nv + v] + (double)xyzi[4 * i + 3];
    out[1 * nv + v] = out[1 * nv + v] + (double)sqrtf(x * x + y * y + z * z);
    if (refl) out[2 * nv + v] = out[2 * nv + v] + (double)refl[i];
    if (amb) out[3 * nv + v] = out[3 * nv + v] + (double)amb[i];
    hist[v] = hist[v] + 1;
  }
  for (int c = 0; c < 4; ++c)
    for (size_t v = 0; v < nv; ++v) {
      const double q = out[c * nv + v] / hist[v];
      out[c * nv + v] = isfinite(q) ? q : 0.0;
    }
  free(hist);
  free(lin);
}

/* ------------------------------------------------------------------------ */
/* Spatial correlation (spatial-correlation.cc:11-206,                       */
/* spatial-correlation-laplace.cc:17-89).  r2c_3d(N,N,N): half spectrum of   */
/* N*N*(N/2+1) entries, linear index (kz*N + kx)*(N/2+1) + ky.  The c2r       */
/* takes Re(sum over the half spectrum with weight 1 on ky = 0 and the       */
/* Nyquist plane, 2 elsewhere) -- FFTW's c2r on a half spectrum.            */
/* ------------------------------------------------------------------------ */

static void r2c3d(const double* f, int N, cplx* half) {
  const size_t nv = (size_t)N * N * N;
  const int H2 = N / 2 + 1;
  cplx* a = (cplx*)malloc(sizeof(cplx) * nv);
  for (size_t i = 0; i < nv; ++i) {
    a[i].re = f[i];
    a[i].im = 0.0;
  }
  fft3d(a, N, N, N, -1);
  for (size_t r = 0; r < (size_t)N * N; ++r)
    for (int ky = 0; ky < H2; ++ky) half[r * H2 + ky] = a[r * N + ky];
  free(a);
}

static void c2r3d(const cplx* half, int N, double* out) {
  const size_t nv = (size_t)N * N * N;
  const int H2 = N / 2 + 1;
  cplx* a = (cplx*)calloc(nv, sizeof(cplx));
  for (size_t r = 0; r < (size_t)N * N; ++r)
    for (int ky = 0; ky < H2; ++ky) {
      const int w = (ky == 0 || (N % 2 == 0 && ky == N / 2)) ? 1 : 2;
      a[r * N + ky].re = w * half[r * H2 + ky].re;
      a[r * N + ky].im = w * half[r * H2 + ky].im;
    }
  fft3d(a, N, N, N, +1);
  for (size_t i = 0; i < nv; ++i) out[i] = a[i].re;
  free(a);
}

/* C channels per side, each N^3 doubles.  laplace = 0: plain
 * SpatialCorrelation on channel 0; laplace = 1: fused. */
void orc_spatial_correlation(int N, int C, const double* f, const double* g,
                             int laplace, int levels, double* out) {
  const size_t nv = (size_t)N * N * N;
  const size_t H = (size_t)N * N * (N / 2 + 1);
  cplx* F = (cplx*)malloc(sizeof(cplx) * H * (laplace ? C : 1));
  cplx* G = (cplx*)malloc(sizeof(cplx) * H * (laplace ? C : 1));
  const int nch = laplace ? C : 1;
  for (int c = 0; c < nch; ++c) {
    r2c3d(f + nv * c, N, F + H * c);
    r2c3d(g + nv * c, N, G + H * c);
  }
  cplx* Cc = (cplx*)malloc(sizeof(cplx) * H);
  cplx* vf = (cplx*)malloc(sizeof(cplx) * nch);
  cplx* vg = (cplx*)malloc(sizeof(cplx) * nch);
  for (size_t k = 0; k < H; ++k) {
    cplx a, b;
    if (laplace) {
      const uint32_t p = (uint32_t)((k + (nv >> 1)) % nv);
      const int rule = orc_fusion_rule(p, (uint32_t)nv, levels, 4.0f);
      for (int c = 0; c < nch; ++c) {
        vf[c] = F[H * c + k];
        vg[c] = G[H * c + k];
      }
      a = fuse_at(vf, nch, rule);
      b = fuse_at(vg, nch, rule);
    } else {
      a = F[k];
      b = G[k];
    }
    Cc[k].re = a.re * b.re - a.im * (-b.im);
    Cc[k].im = a.re * (-b.im) + a.im * b.re;
  }
  c2r3d(Cc, N, out);
  free(F);
  free(G);
  free(Cc);
  free(vf);
  free(vg);
}

/* ------------------------------------------------------------------------ */
/* Low-pass variants, restated literally with the reference's shifts.        */
/* ------------------------------------------------------------------------ */

/* SignalUtils::FFTShift / IFFTShift (signal-utils.h:29-47): std::rotate.   */
static void orc_rotate_left(cplx* a, size_t n, size_t s) {
  if (n == 0 || s % n == 0) return;
  s %= n;
  cplx* t = (cplx*)malloc(sizeof(cplx) * n);
  for (size_t i = 0; i < n; ++i) t[i] = a[(i + s) % n];
  memcpy(a, t, sizeof(cplx) * n);
  free(t);
}
static void orc_fftshift_c(cplx* a, size_t n) { orc_rotate_left(a, n, (n % 2 == 0) ? (n >> 1) : (n >> 1) + 1); }
static void orc_ifftshift_c(cplx* a, size_t n) { orc_rotate_left(a, n, n >> 1); }

/* SphericalCorrelationLowPass::correlateSampledSignals (spherical-          */
/* correlation-low-pass.cc:14-59): channel 0, coefficients shifted, zeroed   */
/* outside [lower, upper) (both clipped to B^2), shifted back, correlated.   */
void orc_spherical_correlation_lowpass(int bw, int bw_out, const double* f, const double* g, uint32_t lower,
                                       uint32_t upper, double* corr) {
  const size_t nc = (size_t)bw * bw;
  double *fr = (double*)malloc(sizeof(double) * nc), *fi = (double*)malloc(sizeof(double) * nc);
  double *gr = (double*)malloc(sizeof(double) * nc), *gi = (double*)malloc(sizeof(double) * nc);
  orc_sht(f, bw, fr, fi);
  orc_sht(g, bw, gr, gi);
  cplx* F = (cplx*)malloc(sizeof(cplx) * nc);
  cplx* G = (cplx*)malloc(sizeof(cplx) * nc);
  for (size_t k = 0; k < nc; ++k) {
    F[k].re = fr[k];
    F[k].im = fi[k];
    G[k].re = gr[k];
    G[k].im = gi[k];
  }
  const size_t lo = lower < nc ? lower : nc, hi = upper < nc ? upper : nc;
  orc_fftshift_c(F, nc);
  orc_fftshift_c(G, nc);
  for (size_t i = 0; i < lo; ++i) F[i].re = F[i].im = G[i].re = G[i].im = 0.0;
  for (size_t i = hi; i < nc; ++i) F[i].re = F[i].im = G[i].re = G[i].im = 0.0;
  orc_ifftshift_c(F, nc);
  orc_ifftshift_c(G, nc);
  for (size_t k = 0; k < nc; ++k) {
    fr[k] = F[k].re;
    fi[k] = F[k].im;
    gr[k] = G[k].re;
    gi[k] = G[k].im;
  }
  const int n = 2 * bw_out;
  const size_t nv = (size_t)n * n * n;
  double* vol = (double*)malloc(sizeof(double) * 2 * nv);
  orc_so3_correlate(bw, bw_out, fr, fi, gr, gi, vol);
  for (size_t i = 0; i < nv; ++i) corr[i] = vol[2 * i] * vol[2 * i] + vol[2 * i + 1] * vol[2 * i + 1];
  free(vol);
  free(fr);
  free(fi);
  free(gr);
  free(gi);
  free(F);
  free(G);
}

/* SpatialCorrelationLowPass::correlateSignals (spatial-correlation-low-     */
/* pass.cc:40-90): channel 1; the N^3-long half-spectrum buffers are         */
/* FFT-shifted, the product is formed at Sub2Ind(i, j, k) for i, j, k in     */
/* [lower, upper] (indices beyond N^3, where the reference's CHECK aborts,   */
/* are skipped; the product buffer starts at zero), shifted back, inverted.  */
void orc_spatial_correlation_lowpass(int N, const double* f1, const double* g1, uint32_t lower, uint32_t upper,
                                     double* out) {
  const size_t nv = (size_t)N * N * N;
  cplx* F = (cplx*)calloc(nv, sizeof(cplx));
  cplx* G = (cplx*)calloc(nv, sizeof(cplx));
  r2c3d(f1, N, F);
  r2c3d(g1, N, G);
  orc_fftshift_c(F, nv);
  orc_fftshift_c(G, nv);
  cplx* Cc = (cplx*)calloc(nv, sizeof(cplx));
  for (uint32_t i = lower; i <= upper; ++i)
    for (uint32_t j = lower; j <= upper; ++j)
      for (uint32_t k = lower; k <= upper; ++k) {
        const uint64_t idx = (uint64_t)(i * (uint32_t)N + j) + (uint64_t)N * N * k;
        if (idx >= nv) continue;
        Cc[idx].re = F[idx].re * G[idx].re - F[idx].im * (-G[idx].im);
        Cc[idx].im = F[idx].re * (-G[idx].im) + F[idx].im * G[idx].re;
      }
  orc_ifftshift_c(Cc, nv);
  c2r3d(Cc, N, out);
  free(F);
  free(G);
  free(Cc);
}

/* ComputeTranslationFromIndex (translation-utils.cc:40-52). */
double orc_translation_from_index(double index, uint32_t n_voxels, int lo,
                                  int hi) {
  if (index == 0) return 0.0;
  const double half = n_voxels / 2.0;
  const double width = (double)(abs(lo) + abs(hi) + 1);
  if (index <= half) return index * width / n_voxels;
  return (index - n_voxels) * width / n_voxels;
}

/* ------------------------------------------------------------------------ */
/* Full SphOptRegistration::registerPointCloud (sph-opt-registration.cc:     */
/* 34-95): target = prev (f), source = cur (h).                              */
/* ------------------------------------------------------------------------ */

typedef struct {
  uint32_t rot_bin;
  double rot_peak;
  double zyz[3];
  double quat[4];
  double xyz[3];
  uint32_t voxel;
  double trans_peak;
  double trans[3];
} orc_pose;

/* ------------------------------------------------------------------------ */
/* Peak neighbourhoods (bingham_/gaussian_peak_neighbors > 0).               */
/* ------------------------------------------------------------------------ */

/* GaussianPeakBasedEval::calculateStartEndNeighbor (gaussian-peak-based-    */
/* eval.cc:31-41): [start, end] around index, one-sided near the ends.       */
void orc_peak_window(uint32_t index, uint32_t n, uint32_t k, uint32_t* first, uint32_t* count) {
  const uint32_t start = (k > index) ? index : index - k;
  const uint32_t end = ((uint64_t)k + index >= n) ? index : index + k;
  *first = start;
  *count = end - start + 1u;
}

/* Symmetric eigenproblem by classical Jacobi (largest off-diagonal pivot).  */
static void orc_sym_eig(int n, const double* A0, double* w, double* V) {
  double A[64];
  for (int i = 0; i < n * n; ++i) A[i] = A0[i];
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) V[i * n + j] = (i == j) ? 1.0 : 0.0;
  for (int it = 0; it < 500; ++it) {
    int p = 0, q = 1;
    double big = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = i + 1; j < n; ++j)
        if (fabs(A[i * n + j]) > big) {
          big = fabs(A[i * n + j]);
          p = i;
          q = j;
        }
    if (big < 1e-300) break;
    const double phi = 0.5 * atan2(2.0 * A[p * n + q], A[q * n + q] - A[p * n + p]);
    const double c = cos(phi), s = sin(phi);
    for (int k = 0; k < n; ++k) {
      const double kp = A[k * n + p], kq = A[k * n + q];
      A[k * n + p] = c * kp - s * kq;
      A[k * n + q] = s * kp + c * kq;
    }
    for (int k = 0; k < n; ++k) {
      const double pk = A[p * n + k], qk = A[q * n + k];
      A[p * n + k] = c * pk - s * qk;
      A[q * n + k] = s * pk + c * qk;
    }
    for (int k = 0; k < n; ++k) {
      const double kp = V[k * n + p], kq = V[k * n + q];
      V[k * n + p] = c * kp - s * kq;
      V[k * n + q] = s * kp + c * kq;
    }
  }
  for (int i = 0; i < n; ++i) w[i] = A[i * n + i];
}

/* BinghamPeakBasedEval::retrievePeakNeighbors + Bingham::fit / fitToMoment  */
/* (bingham-peak-based-eval.cc:59-91, bingham.cc:239-295): moment matrix of  */
/* the weighted bin quaternions, its eigenvalues sorted ascending and        */
/* normalised (omega), the mode = eigenvector of the largest one (w >= 0).   */
int orc_bingham_peak(const double* values, uint32_t first, uint32_t count, uint32_t bw, double* mode,
                     double* omega, double* xyz) {
  double sum = 0.0;
  for (uint32_t i = 0; i < count; ++i) sum += values[i];
  if (count > 1 && !(sum > 0.0)) return -1;
  double C[16] = {0};
  for (uint32_t i = 0; i < count; ++i) {
    double zyz[3], q[4];
    orc_bin_to_zyz(first + i, bw, zyz);
    orc_zyz_to_quat(zyz, q);
    const double w = (count > 1) ? values[i] / sum : values[i];
    for (int r = 0; r < 4; ++r)
      for (int c = 0; c < 4; ++c) C[r * 4 + c] += q[r] * w * q[c];
  }
  for (int r = 0; r < 4; ++r)
    for (int c = r + 1; c < 4; ++c) C[r * 4 + c] = C[c * 4 + r] = 0.5 * (C[r * 4 + c] + C[c * 4 + r]);
  double ev[4], V[16];
  orc_sym_eig(4, C, ev, V);
  int idx[4] = {0, 1, 2, 3};
  for (int a = 0; a < 4; ++a)
    for (int b = a + 1; b < 4; ++b)
      if (ev[idx[b]] < ev[idx[a]]) {
        const int t = idx[a];
        idx[a] = idx[b];
        idx[b] = t;
      }
  double tot = ev[0] + ev[1] + ev[2] + ev[3];
  for (int i = 0; i < 4; ++i) omega[i] = tot != 0.0 ? ev[idx[i]] / tot : 0.0;
  const int m = idx[3];
  double nrm = 0.0;
  for (int r = 0; r < 4; ++r) nrm += V[r * 4 + m] * V[r * 4 + m];
  nrm = sqrt(nrm);
  const double sg = V[0 * 4 + m] < 0 ? -1.0 : 1.0;
  for (int r = 0; r < 4; ++r) mode[r] = sg * V[r * 4 + m] / nrm;
  orc_quat_to_xyz(mode, xyz);
  return 0;
}

/* GaussianPeakBasedEval::retrievePeakNeighbors + Gaussian::setMeanAndCov    */
/* (gaussian-peak-based-eval.cc:73-101, gaussian.cc:47-55).                  */
int orc_gaussian_peak(const double* values, uint32_t first, uint32_t count, uint32_t N, int lo, int hi,
                      double* mean, double* cov) {
  double sum = 0.0;
  for (uint32_t i = 0; i < count; ++i) sum += values[i];
  if (!(sum > 0.0)) return -1;
  double* t = (double*)malloc(sizeof(double) * 3 * count);
  for (int a = 0; a < 3; ++a) mean[a] = 0.0;
  for (uint32_t i = 0; i < count; ++i) {
    uint32_t sub[3];
    orc_ind2sub(first + i, N, N, sub);
    for (int a = 0; a < 3; ++a) {
      t[3 * i + a] = orc_translation_from_index((double)sub[a], N, lo, hi);
      mean[a] += t[3 * i + a] * (values[i] / sum);
    }
  }
  for (int k = 0; k < 9; ++k) cov[k] = 0.0;
  for (uint32_t i = 0; i < count; ++i) {
    const double sw = sqrt(values[i] / sum);
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) cov[r * 3 + c] += (t[3 * i + r] - mean[r]) * sw * (t[3 * i + c] - mean[c]) * sw;
  }
  free(t);
  return 0;
}

void orc_register_pair_k(const float* tgt_xyzi, size_t Pt, const float* tgt_refl,
                         const float* src_xyzi, size_t Ps, const float* src_refl,
                         int bw, int N, int lo, int hi, float max_sq_dist, uint32_t rot_k, uint32_t trans_k,
                         orc_pose* pose, double* rot_corr, double* trans_corr, double* omega, double* cov);
void orc_register_pair_mode(const float* tgt_xyzi, size_t Pt, const float* tgt_refl,
                            const float* src_xyzi, size_t Ps, const float* src_refl,
                            int bw, int N, int lo, int hi, float max_sq_dist, uint32_t rot_k, uint32_t trans_k,
                            int sph_mode, orc_pose* pose, double* rot_corr, double* trans_corr, double* omega,
                            double* cov);

void orc_register_pair(const float* tgt_xyzi, size_t Pt, const float* tgt_refl,
                       const float* src_xyzi, size_t Ps, const float* src_refl,
                       int bw, int N, int lo, int hi, float max_sq_dist,
                       orc_pose* pose, double* rot_corr, double* trans_corr) {
  double omega[4], cov[9];
  orc_register_pair_k(tgt_xyzi, Pt, tgt_refl, src_xyzi, Ps, src_refl, bw, N, lo, hi, max_sq_dist, 0, 0, pose,
                      rot_corr, trans_corr, omega, cov);
}

void orc_register_pair_k(const float* tgt_xyzi, size_t Pt, const float* tgt_refl,
                         const float* src_xyzi, size_t Ps, const float* src_refl,
                         int bw, int N, int lo, int hi, float max_sq_dist, uint32_t rot_k, uint32_t trans_k,
                         orc_pose* pose, double* rot_corr, double* trans_corr, double* omega, double* cov) {
  orc_register_pair_mode(tgt_xyzi, Pt, tgt_refl, src_xyzi, Ps, src_refl, bw, N, lo, hi, max_sq_dist, rot_k,
                         trans_k, 0, pose, rot_corr, trans_corr, omega, cov);
}

/* SphericalCorrelation::retrieveInterpolation (spherical-correlation.cc:
 * 103-112): one signal 0.6 * intensity + 0.4 * range per direction, from the
 * sample channels {range, intensity, ...} of n directions. */
void orc_mix_signal(const double* samples, size_t n, double* out) {
  for (size_t i = 0; i < n; ++i) out[i] = 0.6 * samples[n + i] + 0.4 * samples[i];
}

/* With rot_k / trans_k > 0 the rotation applied to the source is the mode    */
/* of the Bingham fit and the translation the mean of the Gaussian fit        */
/* (sph-opt-registration.cc:58-88).  sph_mode 0: SphOptRegistration (4        */
/* channels, Laplace fusion); 1: SphRegistration (sph-registration.cc:166-198: */
/* the single 0.6 I + 0.4 R signal, plain SphericalCorrelation).              */
void orc_register_pair_mode(const float* tgt_xyzi, size_t Pt, const float* tgt_refl,
                            const float* src_xyzi, size_t Ps, const float* src_refl,
                            int bw, int N, int lo, int hi, float max_sq_dist, uint32_t rot_k, uint32_t trans_k,
                            int sph_mode, orc_pose* pose, double* rot_corr, double* trans_corr, double* omega,
                            double* cov) {
  const size_t ns = (size_t)4 * bw * bw;
  double* f = (double*)malloc(sizeof(double) * 4 * ns);
  double* h = (double*)malloc(sizeof(double) * 4 * ns);
  orc_sample_cloud(tgt_xyzi, Pt, tgt_refl, NULL, bw, max_sq_dist, f, NULL);
  orc_sample_cloud(src_xyzi, Ps, src_refl, NULL, bw, max_sq_dist, h, NULL);
  const int n = 2 * bw;
  const size_t nvol = (size_t)n * n * n;
  double* corr = rot_corr ? rot_corr : (double*)malloc(sizeof(double) * nvol);
  if (sph_mode == 1) {
    double* fm = (double*)malloc(sizeof(double) * ns);
    double* hm = (double*)malloc(sizeof(double) * ns);
    orc_mix_signal(f, ns, fm);
    orc_mix_signal(h, ns, hm);
    orc_spherical_correlation(bw, bw, 1, fm, hm, 5, corr, NULL, NULL);
    free(fm);
    free(hm);
  } else {
    orc_spherical_correlation(bw, bw, 4, f, h, 5, corr, NULL, NULL);
  }
  const uint64_t bin = orc_argmax(corr, nvol);
  pose->rot_bin = (uint32_t)bin;
  pose->rot_peak = corr[bin];
  orc_bin_to_zyz((uint32_t)bin, (uint32_t)bw, pose->zyz);
  orc_zyz_to_quat(pose->zyz, pose->quat);
  orc_quat_to_xyz(pose->quat, pose->xyz);
  omega[0] = omega[1] = omega[2] = 0.0;
  omega[3] = 1.0;
  if (rot_k > 0) {
    uint32_t first, count;
    orc_peak_window((uint32_t)bin, (uint32_t)nvol, rot_k, &first, &count);
    orc_bingham_peak(corr + first, first, count, (uint32_t)bw, pose->quat, omega, pose->xyz);
  }
  float T[12];
  orc_rotation_xyz((float)pose->xyz[0], (float)pose->xyz[1], (float)pose->xyz[2], T);
  float* rot = (float*)malloc(sizeof(float) * 4 * (Ps ? Ps : 1));
  memcpy(rot, src_xyzi, sizeof(float) * 4 * Ps);
  orc_transform(rot, Ps, T);
  const size_t nv = (size_t)N * N * N;
  double* fv = (double*)malloc(sizeof(double) * 4 * nv);
  double* gv = (double*)malloc(sizeof(double) * 4 * nv);
  orc_discretize(tgt_xyzi, Pt, tgt_refl, NULL, N, lo, hi, fv);
  orc_discretize(rot, Ps, src_refl, NULL, N, lo, hi, gv);
  double* tc = trans_corr ? trans_corr : (double*)malloc(sizeof(double) * nv);
  orc_spatial_correlation(N, 4, fv, gv, 1, 5, tc);
  const uint64_t vox = orc_argmax(tc, nv);
  pose->voxel = (uint32_t)vox;
  pose->trans_peak = tc[vox];
  uint32_t xyz[3];
  orc_ind2sub((uint32_t)vox, (uint32_t)N, (uint32_t)N, xyz);
  for (int a = 0; a < 3; ++a)
    pose->trans[a] = orc_translation_from_index((double)xyz[a], (uint32_t)N, lo, hi);
  for (int k = 0; k < 9; ++k) cov[k] = 0.0;
  if (trans_k > 0) {
    uint32_t first, count;
    orc_peak_window((uint32_t)vox, (uint32_t)nv, trans_k, &first, &count);
    orc_gaussian_peak(tc + first, first, count, (uint32_t)N, lo, hi, pose->trans, cov);
  }
  if (!rot_corr) free(corr);
  if (!trans_corr) free(tc);
  free(f);
  free(h);
  free(rot);
  free(fv);
  free(gv);
}

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ---------------------------------------------------------------- ingest
 * Voxel-grid downsampling: pcl::VoxelGrid<pcl::PointXYZI>::applyFilter
 * (PCL 1.8.1, absent from the reference tree; called by
 * phaser_pre/src/commands/voxel-grid-cmd.cc:11-22 with leaf
 * --phaser_voxel_grid_leaf_size) restated from PCL's published algorithm in
 * float arithmetic:
 *   bounds of x, y, z over finite points; inv = 1/leaf;
 *   d = int64((max - min) * inv) + 1, output = input when dx*dy*dz > INT32_MAX;
 *   min_b = int(floor(min * inv)), div_b = int(floor(max * inv)) - min_b + 1;
 *   leaf = sum_a int(floor(p_a * inv_a) - float(min_b_a)) * (1, div_x, div_x*div_y)_a;
 *   sort by leaf (stable here: PCL's std::sort leaves the order inside a leaf
 *   unspecified), float sums of x, y, z, intensity in that order, / float(count);
 *   leaves with fewer than min_pts points dropped.
 * Returns the output count, or -1 where PCL's int arithmetic is undefined
 * (floor(coordinate / leaf) outside int32, more than 2^30 leaves along an
 * axis, or more than 2^32 - 1 cells).  Non-finite points are dropped. */
typedef struct {
  uint32_t key, idx;
} orc_leaf_pt;

static int orc_cmp_leaf_pt(const void* a, const void* b) {
  const orc_leaf_pt* x = (const orc_leaf_pt*)a;
  const orc_leaf_pt* y = (const orc_leaf_pt*)b;
  if (x->key != y->key) return x->key < y->key ? -1 : 1;
  return x->idx < y->idx ? -1 : (x->idx > y->idx);
}

int64_t orc_voxel_grid(const float* xyzi, const float* refl, const float* amb, size_t n, float lx, float ly,
                       float lz, uint32_t min_pts, float* out, float* out_refl, float* out_amb) {
  const float inv[3] = {1.0f / lx, 1.0f / ly, 1.0f / lz};
  float mn[3] = {0, 0, 0}, mx[3] = {0, 0, 0};
  size_t n_fin = 0;
  for (size_t i = 0; i < n; ++i) {
    const float* p = xyzi + 4 * i;
    if (!isfinite(p[0]) || !isfinite(p[1]) || !isfinite(p[2])) continue;
    for (int a = 0; a < 3; ++a) {
      if (n_fin == 0 || p[a] < mn[a]) mn[a] = p[a];
      if (n_fin == 0 || p[a] > mx[a]) mx[a] = p[a];
    }
    ++n_fin;
  }
  if (n_fin == 0) return 0;
  int overflow = 0, range = 0;
  long long d[3], div[3];
  int32_t min_b[3];
  for (int a = 0; a < 3; ++a) {
    const float ext = (mx[a] - mn[a]) * inv[a];
    if (!(ext < 4.0e18f)) {
      overflow = 1;
      d[a] = 0;
    } else {
      d[a] = (long long)ext + 1;
    }
    const float fl = floorf(mn[a] * inv[a]), fh = floorf(mx[a] * inv[a]);
    if (!(fl >= -2147483648.0f && fh < 2147483648.0f)) range = 1;
    min_b[a] = range ? 0 : (int32_t)fl;
    div[a] = range ? 1 : (long long)(int32_t)fh - (long long)(int32_t)fl + 1;
    if (div[a] > (1ll << 30)) range = 1;
  }
  if (!overflow) {
    if (d[0] > 2147483647ll || d[1] > 2147483647ll || d[2] > 2147483647ll) overflow = 1;
    else if (d[0] * d[1] > 2147483647ll) overflow = 1;
    else overflow = d[0] * d[1] * d[2] > 2147483647ll;
  }
  if (overflow) {
    memcpy(out, xyzi, sizeof(float) * 4 * n);
    if (refl && out_refl) memcpy(out_refl, refl, sizeof(float) * n);
    if (amb && out_amb) memcpy(out_amb, amb, sizeof(float) * n);
    return (int64_t)n;
  }
  if (range || (unsigned long long)div[0] * (unsigned long long)div[1] * (unsigned long long)div[2] > 0xffffffffull)
    return -1;
  const uint32_t mul[3] = {1u, (uint32_t)div[0], (uint32_t)div[0] * (uint32_t)div[1]};
  orc_leaf_pt* v = (orc_leaf_pt*)malloc(sizeof(orc_leaf_pt) * (n_fin ? n_fin : 1));
  size_t m = 0;
  for (size_t i = 0; i < n; ++i) {
    const float* p = xyzi + 4 * i;
    if (!isfinite(p[0]) || !isfinite(p[1]) || !isfinite(p[2])) continue;
    uint32_t key = 0;
    for (int a = 0; a < 3; ++a) {
      const int32_t ijk = (int32_t)(floorf(p[a] * inv[a]) - (float)min_b[a]);
      key += (uint32_t)ijk * mul[a];
    }
    v[m].key = key;
    v[m].idx = (uint32_t)i;
    ++m;
  }
  qsort(v, m, sizeof(orc_leaf_pt), orc_cmp_leaf_pt);
  int64_t k = 0;
  for (size_t b = 0; b < m;) {
    size_t e = b + 1;
    while (e < m && v[e].key == v[b].key) ++e;
    if (e - b >= min_pts) {
      float s[6] = {0, 0, 0, 0, 0, 0};
      for (size_t j = b; j < e; ++j) {
        const float* p = xyzi + 4 * (size_t)v[j].idx;
        for (int c = 0; c < 4; ++c) s[c] += p[c];
        if (refl) s[4] += refl[v[j].idx];
        if (amb) s[5] += amb[v[j].idx];
      }
      const float cnt = (float)(uint32_t)(e - b);
      for (int c = 0; c < 4; ++c) out[4 * k + c] = s[c] / cnt;
      if (refl && out_refl) out_refl[k] = s[4] / cnt;
      if (amb && out_amb) out_amb[k] = s[5] / cnt;
      ++k;
    }
    b = e;
  }
  free(v);
  return k;
}

/* ---------------------------------------------------------------- padding
 * Zero-padded spatial correlation, restated literally from
 * SpatialCorrelation (spatial-correlation.cc:11-45 constructor, 78-83
 * complexMulSeq, 142-161 complexMulSeqUsingIndices, 163-206 correlateSignals,
 * 223-230 computeZeroPaddedIndex), SpatialCorrelationLaplace
 * (spatial-correlation-laplace.cc:17-89) and SpatialCorrelationLowPass
 * (spatial-correlation-low-pass.cc:40-69), M = N + 2 pad:
 *   state_f / state_g are the reference's F_ / G_ (N^3 complex, re/im
 *   interleaved, zero at construction); each r2c writes their first
 *   N^2 (N/2+1) entries; Laplace and low-pass FFT-shift all N^3 entries,
 *   copy the shifted buffers out per channel; the product of idx goes to
 *   Sub2Ind(i+pad, j+pad, k+pad, M, M) of a zeroed M^3 buffer; Laplace and
 *   low-pass IFFT-shift its first N^3 entries; c2r_3d at M.
 * mode 0 plain (channel 0 of f/g), 1 Laplace (C channels), 2 low-pass
 * (channel 1, cube [lower, upper]^3, indices >= N^3 skipped where the
 * reference aborts).  out: M^3 doubles.  Returns the correlation length the
 * reference reports, uint32(N^3 * ((M / N)^3)) in double. */
uint32_t orc_spatial_correlation_padded(int N, int pad, int C, const double* f, const double* g, int mode,
                                        int levels, uint32_t lower, uint32_t upper, double* state_f,
                                        double* state_g, double* out) {
  const size_t nv = (size_t)N * N * N;
  const int M = N + 2 * pad;
  const size_t nvM = (size_t)M * M * M;
  cplx* Fb = (cplx*)state_f;
  cplx* Gb = (cplx*)state_g;
  cplx* Cc = (cplx*)calloc(nvM, sizeof(cplx));
  const size_t H = (size_t)N * N * (N / 2 + 1);
  cplx* half = (cplx*)malloc(sizeof(cplx) * H);
  const int nch = mode == 1 ? C : 1;
  const int ch0 = mode == 2 ? 1 : 0;
  cplx* Fch = (cplx*)malloc(sizeof(cplx) * nv * nch);
  cplx* Gch = (cplx*)malloc(sizeof(cplx) * nv * nch);
  for (int c = 0; c < nch; ++c) {
    r2c3d(f + nv * (size_t)(ch0 + c), N, half);
    memcpy(Fb, half, sizeof(cplx) * H);
    r2c3d(g + nv * (size_t)(ch0 + c), N, half);
    memcpy(Gb, half, sizeof(cplx) * H);
    if (mode != 0) {
      orc_fftshift_c(Fb, nv);
      orc_fftshift_c(Gb, nv);
    }
    memcpy(Fch + nv * c, Fb, sizeof(cplx) * nv);
    memcpy(Gch + nv * c, Gb, sizeof(cplx) * nv);
  }
  cplx* vf = (cplx*)malloc(sizeof(cplx) * nch);
  cplx* vg = (cplx*)malloc(sizeof(cplx) * nch);
  for (size_t idx = 0; idx < nv; ++idx) {
    const uint32_t j = (uint32_t)(idx % N), i = (uint32_t)((idx / N) % N), k = (uint32_t)(idx / ((size_t)N * N));
    if (mode == 2) {
      /* the index list Sub2Ind(i, j, k, N, N) over the cube; every listed
       * index below N^3 decodes back to its own (i, j, k) when upper < N */
      if (i < lower || i > upper || j < lower || j > upper || k < lower || k > upper) continue;
    }
    cplx a, b;
    if (mode == 1) {
      for (int c = 0; c < nch; ++c) {
        vf[c] = Fch[nv * c + idx];
        vg[c] = Gch[nv * c + idx];
      }
      const int rule = orc_fusion_rule((uint32_t)idx, (uint32_t)nv, levels, 4.0f);
      a = fuse_at(vf, nch, rule);
      b = fuse_at(vg, nch, rule);
    } else {
      a = Fch[idx];
      b = Gch[idx];
    }
    const size_t y = (size_t)(i + pad) * M + (j + pad) + (size_t)M * M * (k + pad);
    Cc[y].re = a.re * b.re - a.im * (-b.im);
    Cc[y].im = a.re * (-b.im) + a.im * b.re;
  }
  if (mode != 0) orc_ifftshift_c(Cc, nv);
  c2r3d(Cc, M, out);
  const double ratio = (double)(uint32_t)M / (double)N;
  const double factor = ratio * ratio * ratio;
  const uint32_t size = (uint32_t)((double)(uint32_t)nv * factor);
  free(Cc);
  free(half);
  free(Fch);
  free(Gch);
  free(vf);
  free(vg);
  return size;
}

/* ZScorePeakExtraction::extractPeaks + calculateSmoothedZScore             */
/* (phaser_core/src/backend/uncertainty/z-score-peak-extraction.cc:42-112):  */
/* a sliding window of `lag` values (mean, standard deviation with divisor  */
/* lag - 1) over a copy of the input; an index above filter_thr that is     */
/* more than thr deviations from the mean is a signal when above it and is  */
/* damped by `influence` before the window moves.  Window sums in index     */
/* order.  Returns the number of signals (indices written to out, at most   */
/* cap of them).                                                            */
uint64_t orc_zscore_peaks(const double* corr, uint64_t n, double lag_pct, uint32_t lag_max, double thr,
                          double influence, double filter_thr, uint32_t* out, uint64_t cap) {
  const uint32_t share = (uint32_t)((double)n * lag_pct);
  const uint64_t lag = share < lag_max ? share : lag_max;
  if (n <= lag + 2) return 0;
  double* in = (double*)malloc(sizeof(double) * n);
  memcpy(in, corr, sizeof(double) * n);
  double avg = 0.0, dev = 0.0, s = 0.0, q = 0.0;
  for (uint64_t k = 0; k < lag; ++k) s += in[k];
  avg = s / (double)lag;
  for (uint64_t k = 0; k < lag; ++k) q += (in[k] - avg) * (in[k] - avg);
  dev = sqrt(q / ((double)lag - 1.0));
  uint64_t count = 0;
  for (uint64_t i = lag + 1; i < n; ++i) {
    const double x = in[i];
    if (x <= filter_thr) continue;
    if (fabs(x - avg) > thr * dev) {
      if (x >= avg) {
        if (count < cap) out[count] = (uint32_t)i;
        ++count;
      }
      in[i] = influence * x + (1.0 - influence) * in[i - 1];
    }
    s = 0.0;
    for (uint64_t k = i - lag; k < i; ++k) s += in[k];
    avg = s / (double)lag;
    q = 0.0;
    for (uint64_t k = i - lag; k < i; ++k) q += (in[k] - avg) * (in[k] - avg);
    dev = sqrt(q / ((double)lag - 1.0));
  }
  free(in);
  return count;
}
