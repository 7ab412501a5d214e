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

// Fused transform: block per (order pair {m, B-1-m}, signal), so every block
// carries B + 1 Legendre degrees.  Phase 1: warps take theta rows k, lanes
// the phi samples j (four loads in flight), and one pass over a row gives
// F_m(theta_k) for both orders.  Phase 2: warps take (order, degree) tasks
// and lanes the rows k of the table.
constexpr int kShtThreads = 1024;

__global__ void __launch_bounds__(kShtThreads) k_sht(int bw, const float* __restrict__ sig,
                                                     const float2* __restrict__ tw, const float* __restrict__ table,
                                                     float2* __restrict__ coef) {
  extern __shared__ float2 sh[];
  const int n = 2 * bw;
  const int m0 = blockIdx.x, m1 = bw - 1 - blockIdx.x;
  const int nm = (m1 > m0) ? 2 : 1;
  float2* twm = sh;          // [2][n] exp(-i m phi_j)
  float2* fk = sh + 2 * n;   // [2][n] F_m(theta_k)
  const int s = blockIdx.y;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    twm[j] = __ldg(&tw[(j * m0) % n]);
    twm[n + j] = __ldg(&tw[(j * m1) % n]);
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const float scale = (float)(2.5066282746310002 / (double)n);  // sqrt(2 pi) / 2B
  const float* S = sig + (size_t)s * n * n;
  for (int k = warp; k < n; k += nw) {
    const float* row = S + (size_t)k * n;
    float ar = 0.f, ai = 0.f, br = 0.f, bi = 0.f;
    for (int j0 = lane; j0 < n; j0 += 128) {
      float v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) v[u] = (j0 + 32 * u < n) ? __ldg(&row[j0 + 32 * u]) : 0.f;
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int j = j0 + 32 * u;
        if (j < n) {
          const float2 w = twm[j], x = twm[n + j];
          ar = fmaf(v[u], w.x, ar);
          ai = fmaf(v[u], w.y, ai);
          br = fmaf(v[u], x.x, br);
          bi = fmaf(v[u], x.y, bi);
        }
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      ar += __shfl_xor_sync(0xffffffffu, ar, o);
      ai += __shfl_xor_sync(0xffffffffu, ai, o);
      br += __shfl_xor_sync(0xffffffffu, br, o);
      bi += __shfl_xor_sync(0xffffffffu, bi, o);
    }
    if (lane == 0) {
      fk[k] = make_float2(ar * scale, ai * scale);
      fk[n + k] = make_float2(br * scale, bi * scale);
    }
  }
  __syncthreads();
  const int nl0 = bw - m0;
  const int ntask = nl0 + (nm == 2 ? bw - m1 : 0);
  for (int task = warp; task < ntask; task += nw) {
    const int h = task < nl0 ? 0 : 1;
    const int m = h ? m1 : m0;
    const int l = m + (h ? task - nl0 : task);
    const float* trow = table + legendre_offset(m, bw) + (size_t)(l - m) * n;
    const float2* f = fk + h * n;
    float ar = 0.f, ai = 0.f;
    for (int k0 = lane; k0 < n; k0 += 128) {
      float t[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) t[u] = (k0 + 32 * u < n) ? __ldg(&trow[k0 + 32 * u]) : 0.f;
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        if (k0 + 32 * u < n) {
          const float2 x = f[k0 + 32 * u];
          ar = fmaf(t[u], x.x, ar);
          ai = fmaf(t[u], x.y, ai);
        }
      }
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
  dim3 g((a.bw + 1) / 2, a.n_sig);
  k_sht<<<g, kShtThreads, (size_t)4 * 2 * a.bw * sizeof(float2), st>>>(a.bw, a.signal, a.tw, a.table, a.coef);
  count_launches(1);
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
  const uint32_t p = ((uint32_t)sean_index(m, l, bw) + (n >> 1)) % n;  // position after FFTShift
  if (a.laplace) op = fusion_op(p, a.bands);
  const bool dropped = a.lowpass && (p < a.lp_lo || p >= a.lp_hi);
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
    if (dropped) r = make_float2(0.f, 0.f);
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
