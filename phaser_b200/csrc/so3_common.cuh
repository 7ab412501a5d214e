// Pieces shared by the SO(3) synthesis kernels (k_so3.cu: FP32 SIMT synthesis;
// k_so3_tc.cu: Wigner-d table and tensor-core synthesis).
//
// Reference behaviour (phaser_core/lib/SOFT/so3_correlate_fftw.c:102-161,
// makeWigner.c:180-210,324-387,634-698, wignerTransforms_fftw.c:407-442):
//   c(l, m1, m2) = 2 pi sqrt(2/(2l+1)) fhat(l, -m1) (-1)^(m1+m2) conj(hhat(l, -m2))
//   S_{m1 m2}(beta_k) = sum_l c(l, m1, m2) dtilde^l_{m1 m2}(beta_k)
// with dtilde the L2-normalised Wigner d, generated by the three-term
// recurrence in l from the seed d^q_{pq}.  One order class (p, q),
// 0 <= p <= q < B, feeds four (m1, m2) outputs of the synthesised half through
//   d_{q p} = (-1)^(q-p) d_{p q},  d_{p,-q}(b) = d_{q,-p}(b) = (-1)^(l+p) d_{p q}(pi - b)
// (the last two are written at the mirrored beta_{2B-1-k}).
#pragma once

#include <math.h>
#include <stdint.h>

#include "common.cuh"

namespace phgpu {

// Recurrence factors for degrees l < bw_in, tabulated on the host once per
// context (so3_wigner_table):
//   b_l = sqrt((2l+3)/(2l+1)) (l+1)(2l+1) / (R(l+1,p) R(l+1,q))
//   a_l = -sqrt((2l+3)/(2l-1)) (l+1)/l R(l,p) R(l,q) / (R(l+1,p) R(l+1,q))
//   g_l = b_l (-p q / (l(l+1))),   R(l,m) = sqrt(l^2 - m^2)
// and the seed's log normalisation from log-factorials.
struct WigTab {
  const double* s1;  // [B+1][B+1] R(l, m) (0 for m >= l)
  const double* r1;  // [B+1][B+1] 1 / R(l, m) (0 for m >= l)
  const double* cl;  // [B+1] sqrt((2l+3)/(2l+1)) (l+1)(2l+1)
  const double* el;  // [B+1] sqrt((2l+3)/(2l-1)) (l+1)/l (l >= 1)
  const double* il;  // [B+1] 1/(l(l+1)) (l >= 1)
  const double* wl;  // [B+1] 2 pi sqrt(2/(2l+1))
  const double* lq;  // [B+1] log((2q+1)/2)
  const double* lf;  // [2B+2] log(k!)
};

__host__ __device__ inline size_t wigner_table_entries(int bw_in) {
  const size_t b1 = (size_t)bw_in + 1;
  return 2 * b1 * b1 + 5 * b1 + 2 * b1;
}

__host__ __device__ inline WigTab wig_tab(const double* t, int bw_in) {
  const size_t b1 = (size_t)bw_in + 1;
  WigTab w;
  w.s1 = t;
  w.r1 = w.s1 + b1 * b1;
  w.cl = w.r1 + b1 * b1;
  w.el = w.cl + b1;
  w.il = w.el + b1;
  w.wl = w.il + b1;
  w.lq = w.wl + b1;
  w.lf = w.lq + b1;
  return w;
}

// Order class c -> (p, q), c = q (q + 1) / 2 + p: classes with the most
// degrees (small q) come first.
__host__ __device__ inline void so3_class(int c, int* p, int* q) {
  int qq = (int)floor((sqrt(8.0 * c + 1.0) - 1.0) * 0.5);
  while ((qq + 1) * (qq + 2) / 2 <= c) ++qq;
  while (qq * (qq + 1) / 2 > c) --qq;
  *q = qq;
  *p = c - qq * (qq + 1) / 2;
}

// Recurrence coefficients of degree l = q + i of class (p, q).
__device__ __forceinline__ void wig_factors(const WigTab& W, int b1, int p, int q, int l, double* fa, double* fb,
                                            double* gs) {
  const double rr = __dmul_rn(__ldg(&W.r1[(l + 1) * b1 + p]), __ldg(&W.r1[(l + 1) * b1 + q]));
  const double b = __dmul_rn(__ldg(&W.cl[l]), rr);
  *fb = b;
  *gs = (l == 0) ? 0.0 : __dmul_rn(__dmul_rn(b, -(double)p * (double)q), __ldg(&W.il[l]));
  *fa = (l == 0) ? 0.0
                 : -__dmul_rn(__dmul_rn(__dmul_rn(__ldg(&W.el[l]), __ldg(&W.s1[l * b1 + p])), __ldg(&W.s1[l * b1 + q])),
                              rr);
}

// Seed log-normalisation of class (p, q):
// 0.5 [log((2q+1)/2) + log((2q)!) - log((q-p)!) - log((q+p)!)]
__device__ __forceinline__ double wig_lnorm(const WigTab& W, int p, int q) {
  return 0.5 * (__ldg(&W.lq[q]) + __ldg(&W.lf[2 * q]) - __ldg(&W.lf[q - p]) - __ldg(&W.lf[q + p]));
}

// d^q_{pq}(beta_k) = exp(lnorm) cos(beta/2)^(q+p) sin(beta/2)^(q-p); btab is
// [3][n]: cos(beta_k), log cos(beta_k / 2), log sin(beta_k / 2).
__device__ __forceinline__ double wig_seed(const double* __restrict__ btab, int n, int k, double lnorm, int p, int q) {
  const double lg = lnorm + (double)(q + p) * __ldg(&btab[n + k]) +
                    (q > p ? (double)(q - p) * __ldg(&btab[2 * n + k]) : 0.0);
  return exp(lg);
}

// d^{l+1} = a d^{l-1} + (b cos beta + g) d^l, evaluated without contraction so
// every kernel that runs it produces the same values.
__device__ __forceinline__ double wig_step(double a, double b, double g, double cb, double dprev, double dcur) {
  return __dadd_rn(__dmul_rn(a, dprev), __dmul_rn(__dadd_rn(__dmul_rn(b, cb), g), dcur));
}

__device__ __forceinline__ float2 so3_fused_at(const float2* __restrict__ fz, int bw, int side, int l, int m) {
  return __ldg(&fz[((size_t)side * bw + l) * (2 * bw - 1) + (m + bw - 1)]);
}

// conj(b) * a * s
__device__ __forceinline__ float2 so3_prod_conj(float2 a, float2 b, float s) {
  return make_float2(s * (a.x * b.x + a.y * b.y), s * (a.y * b.x - a.x * b.y));
}

// The four coefficient vectors of class (p, q) at degree l:
//   v0: (p, q); v1: (q, p); v2: (p, -q) [or (-p, p) when p == q]; v3: (q, -p) [0 when p == q]
// with the d-symmetry signs folded in (v2, v3 are used at the mirrored beta).
__device__ __forceinline__ void so3_coefs(const float2* __restrict__ fz, int bw, int p, int q, int l, float wn,
                                          float2 v[4]) {
  const float spq = ((p + q) & 1) ? -wn : wn;
  const float slp = ((l + p) & 1) ? -1.0f : 1.0f;
  const float2 fmp = so3_fused_at(fz, bw, 0, l, -p);
  const float2 fmq = so3_fused_at(fz, bw, 0, l, -q);
  const float2 hmp = so3_fused_at(fz, bw, 1, l, -p);
  v[0] = so3_prod_conj(fmp, so3_fused_at(fz, bw, 1, l, -q), spq);
  // (q, p) with d_{qp} = (-1)^(q-p) d_{pq}: sign (-1)^(p+q) (-1)^(q-p) = +1
  v[1] = so3_prod_conj(fmq, hmp, wn);
  if (p == q) {
    // (-p, p) in the synthesised half: c(l,-p,p) = w F(l,p) conj(H(l,-p)), d factor (-1)^(l+p)
    v[2] = so3_prod_conj(so3_fused_at(fz, bw, 0, l, p), hmp, wn * slp);
    v[3] = make_float2(0.f, 0.f);
  } else {
    // (p, -q) and (q, -p), conjugated into (-p, q) and (-q, p)
    v[2] = so3_prod_conj(fmp, so3_fused_at(fz, bw, 1, l, q), spq * slp);
    v[3] = so3_prod_conj(fmq, so3_fused_at(fz, bw, 1, l, p), spq * slp);
  }
}

// Writes the four sums of class (p, q) at beta k into the half spectrum
// S[a][b][beta] (a = m1 index in [0, n), b = m2 in [0, n/2), beta fastest).
__device__ __forceinline__ void so3_store(float2* __restrict__ S, int n, int p, int q, int k, const float2 acc[4]) {
  const int Bo = n >> 1;
  const int km = n - 1 - k;
  auto at = [&](int a, int b, int kk) -> float2& { return S[((size_t)a * Bo + b) * n + kk]; };
  at(p, q, k) = acc[0];  // (a = p, b = q)
  if (p == q) {
    if (p > 0) at(n - p, p, km) = acc[2];  // (-p, p) at mirrored beta
  } else if (p == 0) {
    at(q, 0, k) = acc[1];              // (q, 0)
    at(n - q, 0, k) = cconj(acc[1]);   // (-q, 0) = conj((q, 0))
  } else {
    at(q, p, k) = acc[1];              // (q, p)
    at(n - p, q, km) = cconj(acc[2]);  // (-p, q) = conj((p, -q))
    at(n - q, p, km) = cconj(acc[3]);  // (-q, p) = conj((q, -p))
  }
}

}  // namespace phgpu
