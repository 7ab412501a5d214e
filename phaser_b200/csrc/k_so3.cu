// Inverse SO(3) transform of the correlation coefficients, |z|^2 and argmax.
//
// Reference behaviour (phaser_core/lib/SOFT/so3_correlate_fftw.c:102-161 and
// soft_fftw.c:1036-1914 with flag = 1, called from
// phaser_core/src/backend/correlation/spherical-correlation.cc:248-279):
//   c(l, m1, m2) = 2 pi sqrt(2/(2l+1)) fhat(l, -m1) (-1)^(m1+m2) conj(hhat(l, -m2))
//   S_{m1 m2}(beta_k) = sum_l c(l, m1, m2) dtilde^l_{m1 m2}(beta_k)
//   z(beta, alpha, gamma) = (B / pi) (1 / 2B) sum S_{m1 m2}(beta) e^{-i(m1 alpha + m2 gamma)}
// where only one member of each pair (m1, m2) / (-m1, -m2) is synthesised
// (the half H = {m1 > 0, m2 != -m1} + {(-m, m)} + {(0, m2 >= 0)}) and the
// other is its conjugate, so z is real.  Output layout [beta][alpha][gamma].
//
// Design: one block per order class (p, q), 0 <= p <= q < B.  Thread k runs
// the FP64 three-term recurrence of dtilde^l_{p q}(beta_k) in l (the Wigner
// table is never stored) and accumulates in FP32 the four outputs the class
// feeds through the d-symmetries
//   d_{q p} = (-1)^(q-p) d_{p q},  d_{p,-q}(b) = d_{q,-p}(b) = (-1)^(l+p) d_{p q}(pi - b)
// at beta_k and at the mirrored beta_{2B-1-k}.  Only b = m2 >= 0 is kept
// (half spectrum); the gamma transform is a Hermitian complex-to-real one.
#include <math.h>

#include <vector>

#include "fft2.cuh"
#include "kernels.h"

namespace phgpu {

__device__ __forceinline__ float2 fused_at(const float2* __restrict__ fz, int bw, int side, int l, int m) {
  return fz[((size_t)side * bw + l) * (2 * bw - 1) + (m + bw - 1)];
}

// conj(b) * a * s
__device__ __forceinline__ float2 prod_conj(float2 a, float2 b, float s) {
  return make_float2(s * (a.x * b.x + a.y * b.y), s * (a.y * b.x - a.x * b.y));
}

// KB betas per thread (k = t, t + ceil(n / KB), ...): the coefficient loads
// from shared memory serve KB recurrences.
constexpr int kSynthBetas = 4;

// Recurrence factors of the L2-normalised Wigner-d three-term recurrence in
// l for degrees l < bw_in, from square roots tabulated on the host once per
// context (so3_wigner_table), so a block's set-up is loads and products:
//   b_l = sqrt((2l+3)/(2l+1)) (l+1)(2l+1) / (R(l+1,p) R(l+1,q))
//   a_l = -sqrt((2l+3)/(2l-1)) (l+1)/l R(l,p) R(l,q) / (R(l+1,p) R(l+1,q))
//   g_l = b_l (-p q / (l(l+1))),   R(l,m) = sqrt(l^2 - m^2)
// and the seed's log normalisation from log-factorials.
struct WigTab {
  const double* s1;   // [B+1][B+1] R(l, m) (0 for m >= l)
  const double* r1;   // [B+1][B+1] 1 / R(l, m) (0 for m >= l)
  const double* cl;   // [B+1] sqrt((2l+3)/(2l+1)) (l+1)(2l+1)
  const double* el;   // [B+1] sqrt((2l+3)/(2l-1)) (l+1)/l (l >= 1)
  const double* il;   // [B+1] 1/(l(l+1)) (l >= 1)
  const double* wl;   // [B+1] 2 pi sqrt(2/(2l+1))
  const double* lq;   // [B+1] log((2q+1)/2)
  const double* lf;   // [2B+2] log(k!)
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

__global__ void k_so3_synth(int bw_in, int bw_out, const float2* __restrict__ fz, const double* __restrict__ btab,
                            const double* __restrict__ wtab, float2* __restrict__ S) {
  extern __shared__ double sm[];
  double* fa = sm;
  double* fb = fa + bw_in;
  double* gs = fb + bw_in;            // fb * shift
  double* s_lnorm = gs + bw_in;       // one value (slot padded to 16 bytes)
  float2* cv = (float2*)(s_lnorm + 2);  // [4][bw_in]
  const int cidx = blockIdx.x;
  int q = (int)floor((sqrt(8.0 * cidx + 1.0) - 1.0) * 0.5);
  while ((q + 1) * (q + 2) / 2 <= cidx) ++q;
  while (q * (q + 1) / 2 > cidx) --q;
  const int p = cidx - q * (q + 1) / 2;
  const int nl = bw_in - q;
  const double dp = p, dq = q;
  const WigTab W = wig_tab(wtab, bw_in);
  const int b1 = bw_in + 1;
  for (int i = threadIdx.x; i < nl; i += blockDim.x) {
    const int l = q + i;
    const double rr = __ldg(&W.r1[(l + 1) * b1 + p]) * __ldg(&W.r1[(l + 1) * b1 + q]);
    const double b = __ldg(&W.cl[l]) * rr;
    fb[i] = b;
    gs[i] = (l == 0) ? 0.0 : b * (-dp * dq) * __ldg(&W.il[l]);
    fa[i] = (l == 0) ? 0.0 : -__ldg(&W.el[l]) * __ldg(&W.s1[l * b1 + p]) * __ldg(&W.s1[l * b1 + q]) * rr;
    const float wn = (float)__ldg(&W.wl[l]);
    const float spq = ((p + q) & 1) ? -wn : wn;
    const float slp = ((l + p) & 1) ? -1.0f : 1.0f;
    // v0: (p, q)
    cv[0 * bw_in + i] = prod_conj(fused_at(fz, bw_in, 0, l, -p), fused_at(fz, bw_in, 1, l, -q), spq);
    // v1: (q, p) with d_{qp} = (-1)^(q-p) d_{pq}: sign (-1)^(p+q) (-1)^(q-p) = +1
    cv[1 * bw_in + i] = prod_conj(fused_at(fz, bw_in, 0, l, -q), fused_at(fz, bw_in, 1, l, -p), wn);
    if (p == q) {
      // (-p, p) in the synthesised half: c(l,-p,p) = w F(l,p) conj(H(l,-p)), d factor (-1)^(l+p)
      cv[2 * bw_in + i] = prod_conj(fused_at(fz, bw_in, 0, l, p), fused_at(fz, bw_in, 1, l, -p), wn * slp);
      cv[3 * bw_in + i] = make_float2(0.f, 0.f);
    } else {
      // (p, -q) and (q, -p), conjugated into (-p, q) and (-q, p)
      cv[2 * bw_in + i] = prod_conj(fused_at(fz, bw_in, 0, l, -p), fused_at(fz, bw_in, 1, l, q), spq * slp);
      cv[3 * bw_in + i] = prod_conj(fused_at(fz, bw_in, 0, l, -q), fused_at(fz, bw_in, 1, l, p), spq * slp);
    }
  }
  if (threadIdx.x == 0) {
    // seed normalisation: 0.5 [log((2q+1)/2) + log((2q)!) - log((q-p)!) - log((q+p)!)]
    *s_lnorm = 0.5 * (__ldg(&W.lq[q]) + __ldg(&W.lf[2 * q]) - __ldg(&W.lf[q - p]) - __ldg(&W.lf[q + p]));
  }
  __syncthreads();
  const int n = 2 * bw_out;
  const int Bo = bw_out;
  const int stride = (n + kSynthBetas - 1) / kSynthBetas;
  const double lnorm = *s_lnorm;
  for (int k0 = threadIdx.x; k0 < stride; k0 += blockDim.x) {
    double cb[kSynthBetas], dcur[kSynthBetas], dprev[kSynthBetas];
    float2 acc[kSynthBetas][4];
#pragma unroll
    for (int u = 0; u < kSynthBetas; ++u) {
      const int k = min(k0 + u * stride, n - 1);
      cb[u] = __ldg(&btab[k]);
      // d^q_{pq}(beta) = exp(lnorm) cos(beta/2)^(q+p) sin(beta/2)^(q-p)
      const double lg = lnorm + (dq + dp) * __ldg(&btab[n + k]) + (q > p ? (dq - dp) * __ldg(&btab[2 * n + k]) : 0.0);
      dcur[u] = exp(lg);
      dprev[u] = 0.0;
#pragma unroll
      for (int v = 0; v < 4; ++v) acc[u][v] = make_float2(0.f, 0.f);
    }
    for (int i = 0; i < nl; ++i) {
      const float2 c0 = cv[i], c1 = cv[bw_in + i], c2 = cv[2 * bw_in + i], c3 = cv[3 * bw_in + i];
      const double a = fa[i], b = fb[i], g = gs[i];
#pragma unroll
      for (int u = 0; u < kSynthBetas; ++u) {
        const float d = (float)dcur[u];
        acc[u][0].x = fmaf(c0.x, d, acc[u][0].x);
        acc[u][0].y = fmaf(c0.y, d, acc[u][0].y);
        acc[u][1].x = fmaf(c1.x, d, acc[u][1].x);
        acc[u][1].y = fmaf(c1.y, d, acc[u][1].y);
        acc[u][2].x = fmaf(c2.x, d, acc[u][2].x);
        acc[u][2].y = fmaf(c2.y, d, acc[u][2].y);
        acc[u][3].x = fmaf(c3.x, d, acc[u][3].x);
        acc[u][3].y = fmaf(c3.y, d, acc[u][3].y);
        // d^{l+1} = a d^{l-1} + b (cos beta + shift) d^l
        const double dn = a * dprev[u] + fma(b, cb[u], g) * dcur[u];
        dprev[u] = dcur[u];
        dcur[u] = dn;
      }
    }
#pragma unroll
    for (int u = 0; u < kSynthBetas; ++u) {
      const int k = k0 + u * stride;
      if (k >= n) continue;
      const int km = n - 1 - k;
      float2* Sk = S + (size_t)k * n * Bo;
      float2* Sm = S + (size_t)km * n * Bo;
      Sk[(size_t)p * Bo + q] = acc[u][0];  // (a = p, b = q)
      if (p == q) {
        if (p > 0) Sm[(size_t)(n - p) * Bo + p] = acc[u][2];  // (-p, p) at mirrored beta
      } else if (p == 0) {
        Sk[(size_t)q * Bo + 0] = acc[u][1];                     // (q, 0)
        Sk[(size_t)(n - q) * Bo + 0] = cconj(acc[u][1]);        // (-q, 0) = conj((q, 0))
      } else {
        Sk[(size_t)q * Bo + p] = acc[u][1];                     // (q, p)
        Sm[(size_t)(n - p) * Bo + q] = cconj(acc[u][2]);        // (-p, q) = conj((p, -q))
        Sm[(size_t)(n - q) * Bo + p] = cconj(acc[u][3]);        // (-q, p) = conj((q, -p))
      }
    }
  }
}

void so3_wigner_table(int bw_in, std::vector<double>& tab) {
  tab.assign(wigner_table_entries(bw_in), 0.0);
  const WigTab W = wig_tab(tab.data(), bw_in);
  const int b1 = bw_in + 1;
  double* s1 = const_cast<double*>(W.s1);
  double* r1 = const_cast<double*>(W.r1);
  for (int l = 0; l <= bw_in; ++l)
    for (int m = 0; m < l; ++m) {
      const double v = sqrt((double)l * l - (double)m * m);
      s1[l * b1 + m] = v;
      r1[l * b1 + m] = 1.0 / v;
    }
  for (int l = 0; l <= bw_in; ++l) {
    const double dl = l;
    const_cast<double*>(W.cl)[l] = sqrt((2 * dl + 3) / (2 * dl + 1)) * (dl + 1) * (2 * dl + 1);
    const_cast<double*>(W.el)[l] = l > 0 ? sqrt((2 * dl + 3) / (2 * dl - 1)) * (dl + 1) / dl : 0.0;
    const_cast<double*>(W.il)[l] = l > 0 ? 1.0 / (dl * (dl + 1)) : 0.0;
    const_cast<double*>(W.wl)[l] = 2.0 * M_PI * sqrt(2.0 / (2.0 * dl + 1.0));
    const_cast<double*>(W.lq)[l] = log((2.0 * dl + 1.0) / 2.0);
  }
  for (int k = 0; k < 2 * bw_in + 2; ++k) const_cast<double*>(W.lf)[k] = lgamma((double)k + 1.0);
}

void so3_beta_table(int bw_out, double* tab) {
  const int n = 2 * bw_out;
  for (int k = 0; k < n; ++k) {
    const double beta = M_PI * (2.0 * k + 1.0) / (4.0 * bw_out);
    tab[k] = cos(beta);
    tab[n + k] = log(cos(0.5 * beta));
    tab[2 * n + k] = log(sin(0.5 * beta));
  }
}

// Forward DFT over a (alpha) for a tile of b columns at one beta.
template <int NF>
__global__ void k_so3_fft_a(int bw_in, int bw_out, float2* __restrict__ S, FftPlan plan) {
  extern __shared__ float2 tile[];
  constexpr int Wt = 16;
  const int n = NF > 0 ? NF : 2 * bw_out;
  const int Bo = n / 2;
  const int k = blockIdx.y;
  const int b0 = blockIdx.x * Wt;
  const int wt = min(Wt, bw_in - b0);
  float2* Sk = S + (size_t)k * n * Bo;
  // four loads in flight per thread
  for (int e0 = threadIdx.x; e0 < n * Wt; e0 += 4 * blockDim.x) {
    float2 v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int e = e0 + u * blockDim.x;
      const int a = e / Wt, bt = e % Wt;
      // rows with |m1| >= bw_in are not synthesised: read them as zero
      const bool row_ok = (a < bw_in) || (a > n - bw_in);
      v[u] = (e < n * Wt && bt < wt && row_ok) ? Sk[(size_t)a * Bo + b0 + bt] : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (e0 + u * blockDim.x < n * Wt) tile[e0 + u * blockDim.x] = v[u];
  }
  __syncthreads();
  fft_any<NF, false, 4>(tile, Wt, 1, Wt, plan);
  for (int e = threadIdx.x; e < n * Wt; e += blockDim.x) {
    const int a = e / Wt, bt = e % Wt;
    if (bt < wt) Sk[(size_t)a * Bo + b0 + bt] = tile[e];
  }
}

// Hermitian complex-to-real transform over gamma, |z|^2 and argmax.
template <int NF>
__global__ void k_so3_c2r(int bw_in, int bw_out, const float2* __restrict__ S, FftPlan plan,
                          unsigned long long* __restrict__ argmax, float* __restrict__ volume) {
  extern __shared__ float2 rows[];
  constexpr int R = 16;
  const int n = NF > 0 ? NF : 2 * bw_out;
  const int Bo = n / 2;
  const int k = blockIdx.y;
  const int r0 = blockIdx.x * R;
  const int nr = min(R, n - r0);
  int* pos = reinterpret_cast<int*>(rows + R * n);  // [n] positions of gamma frequencies
  int* alpha_of = pos + n;                          // [R] alpha of each row
  for (int e = threadIdx.x; e < R * n; e += blockDim.x) rows[e] = make_float2(0.f, 0.f);
  for (int b = threadIdx.x; b < n; b += blockDim.x) pos[b] = freq2pos<NF>(b, plan);
  for (int r = threadIdx.x; r < nr; r += blockDim.x) alpha_of[r] = pos2freq<NF>(r0 + r, plan);
  __syncthreads();
  for (int e = threadIdx.x; e < nr * Bo; e += blockDim.x) {
    const int r = e / Bo, b = e - r * Bo;
    float2* row = rows + r * n;
    const float2 u = b < bw_in ? S[((size_t)k * n + r0 + r) * Bo + b] : make_float2(0.f, 0.f);
    row[pos[b]] = cconj(u);
    if (b > 0) row[pos[n - b]] = u;
  }
  __syncthreads();
  fft_any<NF, true>(rows, R, n, 1, plan);
  const float K = (float)((1.0 / (double)n) * ((double)Bo / M_PI));
  unsigned long long best = 0ull;
  for (int e = threadIdx.x; e < R * n; e += blockDim.x) {
    const int r = e / n, g = e - r * n;
    if (r < nr) {
      const float v = rows[e].x * K;
      const float v2 = v * v;
      const int alpha = alpha_of[r];
      const uint32_t idx = ((uint32_t)k * n + (uint32_t)alpha) * n + g;
      const unsigned long long key = pack_argmax(v2, idx);
      best = key > best ? key : best;
      if (volume) volume[idx] = v2;
    }
  }
  warp_argmax_commit(best, argmax);
}

// Rows (alpha) of one block of the packed transform: two Hermitian rows per
// complex transform.
template <int NF>
constexpr int c2r_pair_rows() {
  return (NF % 40 == 0) ? 40 : 32;
}

// The same C2R for lengths with a register-tail plan: rows a0 and a1 (two
// alphas) are inverted by one complex transform of Z = X0 + i X1, whose
// output is x0 + i x1 since both spectra are Hermitian.  Row a holds
// X[b] = conj(u_b), X[n - b] = u_b for 0 < b < n/2; its DC term is taken
// real (its imaginary part only ever reaches the imaginary output, which the
// real transform discards) and the Nyquist term is zero, as the
// one-row-per-transform kernel above fills it.
template <int NF>
__global__ void __launch_bounds__(256) k_so3_c2r_tail(int bw_in, const float2* __restrict__ S, FftPlan plan,
                                                     unsigned long long* __restrict__ argmax,
                                                     float* __restrict__ volume) {
  constexpr int n = NF, Bo = NF / 2, RB = c2r_pair_rows<NF>(), ST = NF + 1;
  extern __shared__ float2 zrow[];  // [RB / 2][ST]: one row pair per complex transform
  __shared__ int s_pos[NF];
  __shared__ int s_alpha[RB];
  const int k = blockIdx.y;
  const int r0 = blockIdx.x * RB;
  const int nr = min(RB, n - r0);
  const int np = (nr + 1) >> 1;
  for (int b = threadIdx.x; b < n; b += blockDim.x) s_pos[b] = fixed_freq2pos<NF>(b);
  for (int r = threadIdx.x; r < nr; r += blockDim.x) s_alpha[r] = fixed_pos2freq<NF>(r0 + r);
  __syncthreads();
  const float2* Sk = S + ((size_t)k * n + r0) * Bo;
  constexpr int U = 2;  // pairs of loads in flight per thread
  for (int e0 = threadIdx.x; e0 < np * Bo; e0 += U * blockDim.x) {
    float2 u0[U], u1[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int e = e0 + u * blockDim.x;
      const int p = e / Bo, b = e - p * Bo;
      const bool ok = e < np * Bo && b < bw_in;
      u0[u] = ok ? Sk[(size_t)(2 * p) * Bo + b] : make_float2(0.f, 0.f);
      u1[u] = (ok && 2 * p + 1 < nr) ? Sk[(size_t)(2 * p + 1) * Bo + b] : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int e = e0 + u * blockDim.x;
      if (e >= np * Bo) continue;
      const int p = e / Bo, b = e - p * Bo;
      float2* z = zrow + p * ST;
      if (b == 0) {
        z[s_pos[0]] = make_float2(u0[u].x, u1[u].x);
        z[s_pos[Bo]] = make_float2(0.f, 0.f);
      } else {
        z[s_pos[b]] = make_float2(u0[u].x + u1[u].y, u1[u].x - u0[u].y);      // conj(u0) + i conj(u1)
        z[s_pos[n - b]] = make_float2(u0[u].x - u1[u].y, u0[u].y + u1[u].x);  // u0 + i u1
      }
    }
  }
  __syncthreads();
  fft_tail<NF, true, false>(zrow, np, ST, plan.tw);
  const float K = (float)((1.0 / (double)n) * ((double)Bo / M_PI));
  // per thread: the largest value, the lowest index among equal ones
  float bv = -1.0f;
  uint32_t bi = 0xffffffffu;
  for (int e = threadIdx.x; e < np * n; e += blockDim.x) {
    const int p = e / n, g = e - p * n;
    const float2 z = zrow[p * ST + g];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int r = 2 * p + h;
      if (r < nr) {
        const float v = (h ? z.y : z.x) * K;
        const float v2 = v * v;
        const uint32_t idx = ((uint32_t)k * n + (uint32_t)s_alpha[r]) * n + g;
        if (v2 > bv || (v2 == bv && idx < bi)) {
          bv = v2;
          bi = idx;
        }
        if (volume) volume[idx] = v2;
      }
    }
  }
  warp_argmax_commit(bi == 0xffffffffu ? 0ull : pack_argmax(bv, bi), argmax);
}

template <int NF>
static cudaError_t so3_attrs() {
  const int m = 227 * 1024;
  cudaError_t e = cudaFuncSetAttribute(k_so3_fft_a<NF>, cudaFuncAttributeMaxDynamicSharedMemorySize, m);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_so3_c2r<NF>, cudaFuncAttributeMaxDynamicSharedMemorySize, m);
  if constexpr (Tail<NF>::ok) {
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_so3_c2r_tail<NF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (c2r_pair_rows<NF>() / 2) * (NF + 1) * (int)sizeof(float2));
  }
  return e;
}

cudaError_t so3_init_attributes() {
  cudaError_t e = cudaSuccess;
  for (int n : {64, 128, 200, 256, 320, 512, 0}) {  // every length PHGPU_DISPATCH_N instantiates
    cudaError_t r = cudaSuccess;
    PHGPU_DISPATCH_N(n, r = so3_attrs<NF>());
    if (r != cudaSuccess) e = r;
  }
  return e;
}

cudaError_t launch_so3_synth(const So3Args& a, cudaStream_t st) {
  const int ncls = a.bw_in * (a.bw_in + 1) / 2;
  const int n = 2 * a.bw_out;
  int thr = (((n + kSynthBetas - 1) / kSynthBetas + 31) / 32) * 32;
  if (thr > 512) thr = 512;
  const size_t sm1 = (size_t)a.bw_in * 3 * sizeof(double) + 2 * sizeof(double) + (size_t)a.bw_in * 4 * sizeof(float2);
  k_so3_synth<<<ncls, thr, sm1, st>>>(a.bw_in, a.bw_out, a.fused, a.beta_tab, a.wig_tab, a.S);
  count_launches(1);
  return cudaGetLastError();
}

// The gamma transform: packed pairs on the register-tail engine where the
// length has a tail plan, one row per transform otherwise.
template <int NF>
static void launch_so3_c2r(const So3Args& a, int n, cudaStream_t st) {
  if constexpr (Tail<NF>::ok) {
    constexpr int RB = c2r_pair_rows<NF>();
    dim3 g((n + RB - 1) / RB, n);
    k_so3_c2r_tail<NF><<<g, 256, (size_t)(RB / 2) * (NF + 1) * sizeof(float2), st>>>(a.bw_in, a.S, *a.plan,
                                                                                       a.argmax, a.volume);
  } else {
    dim3 g((n + 15) / 16, n);
    k_so3_c2r<NF><<<g, 256, (size_t)16 * n * sizeof(float2) + (size_t)(n + 16) * sizeof(int), st>>>(
        a.bw_in, a.bw_out, a.S, *a.plan, a.argmax, a.volume);
  }
}

cudaError_t launch_so3_fft(const So3Args& a, cudaStream_t st) {
  const int n = 2 * a.bw_out;
  dim3 g2((a.bw_in + 15) / 16, n);
  PHGPU_DISPATCH_N(n,
      k_so3_fft_a<NF><<<g2, 256, (size_t)n * 16 * sizeof(float2), st>>>(a.bw_in, a.bw_out, a.S, *a.plan);
      launch_so3_c2r<NF>(a, n, st));
  count_launches(2);
  return cudaGetLastError();
}

}  // namespace phgpu
