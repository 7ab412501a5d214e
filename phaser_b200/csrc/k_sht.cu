// Forward spherical-harmonic transform of the sampled S^2 grids and the
// positional Laplace-pyramid fusion of the channel spectra.
//
// Behaviour of SOFT's FST_semi_memo on real data with cutoff = B
// (phaser_core/lib/SOFT/s2_semi_memo.c:123-367): the semi-naive algorithm is an
// exact evaluation of the Driscoll-Healy quadrature
//   F_m(theta_k) = sqrt(2 pi) / (2B) * sum_j f(theta_k, phi_j) exp(-i m phi_j)
//   fhat(l, m)   = sum_k w_k Pbar_l^m(cos theta_k) F_m(theta_k),   0 <= m <= l < B
// with Pbar L2-normalised on [-1, 1] including the Condon-Shortley phase, and
// fhat(l, -m) = (-1)^m conj(fhat(l, m)).  The table w_k Pbar_l^m(cos theta_k)
// is generated once per bandwidth in FP64 by the three-term recurrence in l
// and rounded once to FP32; the transforms themselves run in FP32.
//
// Fusion: SphericalCorrelationLaplace::correlateSampledSignals
// (phaser_core/src/backend/correlation/spherical-correlation-laplace.cc:14-40)
// FFT-shifts each B^2 seanindex-ordered coefficient array, fuses channels with
// LaplacePyramid::fuseChannels (5 levels, divider 4) and shifts back; the
// fused value at coefficient (l, m) therefore follows the positional rule at
// p = (seanindex(m, l) + floor(B^2 / 2)) mod B^2.
#include "kernels.h"

namespace phgpu {

__host__ __device__ inline int sean_index(int m, int l, int bw) {
  const int L = bw - 1;
  if (m >= 0) return m * (L + 1) - ((m * (m - 1)) / 2) + (l - m);
  const int am = -m;
  return ((L * (L + 3)) / 2) + 1 + ((L + m) * (L + m + 1) / 2) + (l - am);
}

size_t legendre_table_entries(int bw) { return (size_t)bw * bw * (bw + 1); }

__host__ __device__ inline size_t legendre_offset(int m, int bw) {
  return (size_t)2 * bw * ((size_t)m * bw - (size_t)m * (m - 1) / 2);
}

// One thread per (m, k): FP64 recurrence over l, rounded once to float.
__global__ void k_legendre_table(int bw, const double* __restrict__ w, float* __restrict__ table) {
  const int n = 2 * bw;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= bw * n) return;
  const int m = idx / n, k = idx % n;
  const double th = M_PI * (2.0 * k + 1.0) / (4.0 * bw);
  const double x = cos(th), s = sin(th);
  // log |Pbar_m^m| = 0.5 log((2m+1)/2) + 0.5 (lgamma(2m+1) - 2 lgamma(m+1) - m log 4) + m log sin
  const double lg = 0.5 * log((2.0 * m + 1.0) / 2.0) +
                    0.5 * (lgamma(2.0 * m + 1.0) - 2.0 * lgamma(m + 1.0) - m * log(4.0)) +
                    (m > 0 ? m * log(s) : 0.0);
  double pcur = exp(lg);
  if (m & 1) pcur = -pcur;
  double pprev = 0.0;
  const double wk = w[k];
  float* out = table + legendre_offset(m, bw) + k;
  out[0] = (float)(wk * pcur);
  for (int l = m; l + 1 < bw; ++l) {
    const double a = sqrt((2.0 * l + 1.0) * (2.0 * l + 3.0) / ((double)(l + 1 - m) * (double)(l + 1 + m)));
    const double b = (l > m) ? sqrt((2.0 * l + 3.0) * (double)(l - m) * (double)(l + m) /
                                    ((2.0 * l - 1.0) * (double)(l + 1 - m) * (double)(l + 1 + m)))
                             : 0.0;
    const double pn = a * x * pcur - b * pprev;
    pprev = pcur;
    pcur = pn;
    out[(size_t)(l + 1 - m) * n] = (float)(wk * pcur);
  }
}

cudaError_t launch_legendre_table(int bw, const double* weights_dev, float* table, cudaStream_t st) {
  const int tot = bw * 2 * bw;
  k_legendre_table<<<(tot + 127) / 128, 128, 0, st>>>(bw, weights_dev, table);
  count_launches(1);
  return cudaGetLastError();
}

// phi DFT: block per (signal, theta row); thread per order m.
__global__ void k_sht_phi(int bw, const float* __restrict__ sig, const float2* __restrict__ tw,
                          float2* __restrict__ fm) {
  extern __shared__ float row[];
  const int n = 2 * bw;
  const int s = blockIdx.y, k = blockIdx.x;
  const float* src = sig + ((size_t)s * n + k) * n;
  for (int j = threadIdx.x; j < n; j += blockDim.x) row[j] = src[j];
  __syncthreads();
  const float scale = (float)(2.5066282746310002 / (double)n);  // sqrt(2 pi) / 2B
  for (int m = threadIdx.x; m < bw; m += blockDim.x) {
    float ar = 0.f, ai = 0.f;
    int t = 0;
    for (int j = 0; j < n; ++j) {
      const float2 w = __ldg(&tw[t]);
      ar = fmaf(row[j], w.x, ar);
      ai = fmaf(row[j], w.y, ai);
      t += m;
      if (t >= n) t -= n;
    }
    fm[((size_t)s * bw + m) * n + k] = make_float2(ar * scale, ai * scale);
  }
}

// Legendre contraction: block per (m, signal); warp per degree l, lanes over k.
__global__ void k_sht_legendre(int bw, const float* __restrict__ table, const float2* __restrict__ fm,
                               float2* __restrict__ coef) {
  extern __shared__ float2 fk[];
  const int n = 2 * bw;
  const int m = blockIdx.x, s = blockIdx.y;
  const float2* src = fm + ((size_t)s * bw + m) * n;
  for (int k = threadIdx.x; k < n; k += blockDim.x) fk[k] = src[k];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const float* tb = table + legendre_offset(m, bw);
  for (int l = m + warp; l < bw; l += nw) {
    const float* trow = tb + (size_t)(l - m) * n;
    float ar = 0.f, ai = 0.f;
    for (int k = lane; k < n; k += 32) {
      const float t = __ldg(&trow[k]);
      ar = fmaf(t, fk[k].x, ar);
      ai = fmaf(t, fk[k].y, ai);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      ar += __shfl_xor_sync(0xffffffffu, ar, o);
      ai += __shfl_xor_sync(0xffffffffu, ai, o);
    }
    if (lane == 0) coef[((size_t)s * bw + l) * bw + m] = make_float2(ar, ai);
  }
}

cudaError_t launch_sht(const ShtArgs& a, cudaStream_t st) {
  const int n = 2 * a.bw;
  dim3 g1(n, a.n_sig);
  k_sht_phi<<<g1, 128, n * sizeof(float), st>>>(a.bw, a.signal, a.tw, a.fm);
  dim3 g2(a.bw, a.n_sig);
  k_sht_legendre<<<g2, 256, n * sizeof(float2), st>>>(a.bw, a.table, a.fm, a.coef);
  count_launches(2);
  return cudaGetLastError();
}

__device__ __forceinline__ float2 coef_at(const float2* __restrict__ c, int bw, int l, int m) {
  const int am = m < 0 ? -m : m;
  float2 v = c[(size_t)l * bw + am];
  if (m < 0) {
    v.y = -v.y;
    if (am & 1) {
      v.x = -v.x;
      v.y = -v.y;
    }
  }
  return v;
}

// One thread per (l, m) with |m| <= l; both sides.
__global__ void k_fuse_s2(FuseS2Args a) {
  const int bw = a.bw;
  const int w = 2 * bw - 1;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= bw * w) return;
  const int l = idx / w, mi = idx % w;
  const int m = mi - (bw - 1);
  if (m > l || -m > l) return;
  const uint32_t n = (uint32_t)(bw * bw);
  int op = kFuseMax;
  if (a.laplace) {
    const uint32_t p = ((uint32_t)sean_index(m, l, bw) + (n >> 1)) % n;
    op = fusion_op(p, a.bands);
  }
  for (int side = 0; side < 2; ++side) {
    const float2* base = a.coef + (size_t)side * a.n_data_ch * bw * bw;
    float2 r = make_float2(0.f, 0.f);
    if (!a.laplace) {
      r = coef_at(base, bw, l, m);
    } else if (op == kFuseMean) {
      float sr = 0.f, si = 0.f;
      for (int c = 0; c < a.n_data_ch; ++c) {
        const float2 v = coef_at(base + (size_t)c * bw * bw, bw, l, m);
        sr += v.x;
        si += v.y;
      }
      r = make_float2(sr / (float)a.n_total_ch, si / (float)a.n_total_ch);
    } else if (op == kFuseMax) {
      float be = -1.0f;
      for (int c = 0; c < a.n_data_ch; ++c) {
        const float2 v = coef_at(base + (size_t)c * bw * bw, bw, l, m);
        const float e = v.x * v.x + v.y * v.y;
        if (e > be) {
          be = e;
          r = v;
        }
      }
    }
    a.fused[((size_t)side * bw + l) * w + mi] = r;
  }
}

cudaError_t launch_fuse_s2(const FuseS2Args& a, cudaStream_t st) {
  const int tot = a.bw * (2 * a.bw - 1);
  k_fuse_s2<<<(tot + 255) / 256, 256, 0, st>>>(a);
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace phgpu
