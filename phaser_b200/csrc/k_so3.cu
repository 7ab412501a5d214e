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
// The half spectrum is laid out S[a][b][beta] (a = m1 index in [0, 2B),
// b = m2 >= 0, beta fastest), so a synthesis thread per beta writes
// coalesced runs and both angle transforms read 128-byte beta segments.
//
// FP32 synthesis (k_so3_synth): one block per order class (p, q),
// 0 <= p <= q < B.  Thread k runs the FP64 three-term recurrence of
// dtilde^l_{p q}(beta_k) in l and accumulates in FP32 the four outputs the
// class feeds (so3_common.cuh).  The tensor-core synthesis from a stored
// Wigner table is in k_so3_tc.cu.  Only b = m2 >= 0 is kept (half spectrum);
// the gamma transform is a Hermitian complex-to-real one.
//
// Every kernel takes a batch of requests (grid dimension z or y): requests of
// one (B, bw_out) shape share the tables and plans.
#include <math.h>

#include <vector>

#include "fft2.cuh"
#include "kernels.h"
#include "so3_common.cuh"

namespace phgpu {

// KB betas per thread (k = t, t + ceil(n / KB), ...): the coefficient loads
// from shared memory serve KB recurrences.
constexpr int kSynthBetas = 4;

__global__ void k_so3_synth(int bw_in, int bw_out, So3Batch bt, const double* __restrict__ btab,
                            const double* __restrict__ wtab) {
  extern __shared__ double sm[];
  double* fa = sm;
  double* fb = fa + bw_in;
  double* gs = fb + bw_in;            // fb * shift
  double* s_lnorm = gs + bw_in;       // one value (slot padded to 16 bytes)
  float2* cv = (float2*)(s_lnorm + 2);  // [4][bw_in]
  const float2* __restrict__ fz = bt.fused[blockIdx.y];
  float2* __restrict__ S = bt.out[blockIdx.y].S;
  int p, q;
  so3_class(blockIdx.x, &p, &q);
  const int nl = bw_in - q;
  const WigTab W = wig_tab(wtab, bw_in);
  const int b1 = bw_in + 1;
  for (int i = threadIdx.x; i < nl; i += blockDim.x) {
    const int l = q + i;
    wig_factors(W, b1, p, q, l, &fa[i], &fb[i], &gs[i]);
    float2 v[4];
    so3_coefs(fz, bw_in, p, q, l, (float)__ldg(&W.wl[l]), v);
#pragma unroll
    for (int u = 0; u < 4; ++u) cv[u * bw_in + i] = v[u];
  }
  if (threadIdx.x == 0) *s_lnorm = wig_lnorm(W, p, q);
  __syncthreads();
  const int n = 2 * bw_out;
  const int stride = (n + kSynthBetas - 1) / kSynthBetas;
  const double lnorm = *s_lnorm;
  for (int k0 = threadIdx.x; k0 < stride; k0 += blockDim.x) {
    double cb[kSynthBetas], dcur[kSynthBetas], dprev[kSynthBetas];
    float2 acc[kSynthBetas][4];
#pragma unroll
    for (int u = 0; u < kSynthBetas; ++u) {
      const int k = min(k0 + u * stride, n - 1);
      cb[u] = __ldg(&btab[k]);
      dcur[u] = wig_seed(btab, n, k, lnorm, p, q);
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
        const double dn = wig_step(a, b, g, cb[u], dprev[u], dcur[u]);
        dprev[u] = dcur[u];
        dcur[u] = dn;
      }
    }
#pragma unroll
    for (int u = 0; u < kSynthBetas; ++u) {
      const int k = k0 + u * stride;
      if (k < n) so3_store(S, n, p, q, k, acc[u]);
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

// Forward DFT over a (alpha) for one b and a tile of Wt = 2^LOG2W betas
// (8, 16 or 32: a tuned parameter, 16 by default).
constexpr int kSo3FftAThreads = 256;
template <int NF, int LOG2W>
__global__ void k_so3_fft_a(int bw_in, int bw_out, So3Batch bt, FftPlan plan) {
  extern __shared__ float2 tile[];  // [a][beta tile]
  constexpr int Wt = 1 << LOG2W;
  const int n = NF > 0 ? NF : 2 * bw_out;
  const int Bo = n / 2;
  const int b = blockIdx.y;
  const int k0 = blockIdx.x * Wt;
  const int wt = min(Wt, n - k0);
  float2* __restrict__ S = bt.out[blockIdx.z].S + (size_t)b * n + k0;
  const size_t astride = (size_t)Bo * n;
  // four loads in flight per thread
  for (int e0 = threadIdx.x; e0 < n * Wt; e0 += 4 * blockDim.x) {
    float2 v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int e = e0 + u * blockDim.x;
      const int a = e / Wt, t = e % Wt;
      // rows with |m1| >= bw_in are not synthesised: read them as zero
      const bool row_ok = (a < bw_in) || (a > n - bw_in);
      v[u] = (e < n * Wt && t < wt && row_ok) ? S[(size_t)a * astride + t] : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (e0 + u * blockDim.x < n * Wt) tile[e0 + u * blockDim.x] = v[u];
  }
  __syncthreads();
  // per-component butterflies (fixed_stage): the packed column-resident form
  // ran about 1 % faster but rounds the SO(3) volume differently, and one
  // near-tied pair of the 256-pair batched workload then picked another bin
  // under the tf32x3 synthesis than under FP32 and the FP64 oracle
  fft_any<NF, false, LOG2W>(tile, Wt, 1, Wt, plan);
  for (int e = threadIdx.x; e < n * Wt; e += blockDim.x) {
    const int a = e / Wt, t = e % Wt;
    if (t < wt) S[(size_t)a * astride + t] = tile[e];
  }
}

// Hermitian complex-to-real transform over gamma, |z|^2 and argmax: one alpha
// row position and a tile of R betas, one beta per transform (lengths without
// a register-tail plan).
template <int NF>
__global__ void k_so3_c2r(int bw_in, int bw_out, So3Batch bt, FftPlan plan) {
  extern __shared__ float2 rows[];  // [R][n]
  constexpr int R = 16;
  const int n = NF > 0 ? NF : 2 * bw_out;
  const int Bo = n / 2;
  const So3Out o = bt.out[blockIdx.z];
  const int r = blockIdx.y;  // alpha row position of the alpha transform's output
  const int k0 = blockIdx.x * R;
  const int nk = min(R, n - k0);
  int* pos = reinterpret_cast<int*>(rows + R * n);  // [n] positions of gamma frequencies
  for (int e = threadIdx.x; e < R * n; e += blockDim.x) rows[e] = make_float2(0.f, 0.f);
  for (int b = threadIdx.x; b < n; b += blockDim.x) pos[b] = freq2pos<NF>(b, plan);
  __syncthreads();
  const int alpha = pos2freq<NF>(r, plan);
  const float2* __restrict__ Sr = o.S + (size_t)r * Bo * n + k0;
  for (int e = threadIdx.x; e < Bo * R; e += blockDim.x) {
    const int b = e / R, j = e - b * R;
    if (j >= nk) continue;
    float2* row = rows + j * n;
    const float2 u = b < bw_in ? Sr[(size_t)b * n + j] : make_float2(0.f, 0.f);
    row[pos[b]] = cconj(u);
    if (b > 0) row[pos[n - b]] = u;
  }
  __syncthreads();
  fft_any<NF, true>(rows, R, n, 1, plan);
  const float K = (float)((1.0 / (double)n) * ((double)Bo / M_PI));
  unsigned long long best = 0ull;
  for (int e = threadIdx.x; e < R * n; e += blockDim.x) {
    const int j = e / n, g = e - j * n;
    if (j < nk) {
      const float v = rows[e].x * K;
      const float v2 = v * v;
      const uint32_t idx = ((uint32_t)(k0 + j) * n + (uint32_t)alpha) * n + g;
      const unsigned long long key = pack_argmax(v2, idx);
      best = key > best ? key : best;
      if (o.volume) o.volume[idx] = v2;
    }
  }
  warp_argmax_commit(best, o.argmax);
}

// Betas of one block of the packed transform: two Hermitian sequences per
// complex transform.
template <int NF>
constexpr int c2r_pair_rows() {
  return (NF % 40 == 0) ? 40 : 32;
}

// The same C2R for lengths with a register-tail plan: betas k and k + 1 of
// one alpha are inverted by one complex transform of Z = X0 + i X1, whose
// output is x0 + i x1 since both spectra are Hermitian.  Sequence X holds
// X[b] = conj(u_b), X[n - b] = u_b for 0 < b < n/2; its DC term is taken real
// (its imaginary part only ever reaches the imaginary output, which the real
// transform discards) and the Nyquist term is zero, as the one-sequence-per-
// transform kernel above fills it.  A pair of betas is one 16-byte load.
// Four blocks per SM (64 registers) rather than the three that 74 registers
// allowed: 0.0488 vs 0.0511 ms for the SO(3) angle transforms at B = 100.
constexpr int kSo3TailThreads = 256;
template <int NF>
__global__ void __launch_bounds__(kSo3TailThreads, 4) k_so3_c2r_tail(int bw_in, So3Batch bt, FftPlan plan) {
  constexpr int n = NF, Bo = NF / 2, RB = c2r_pair_rows<NF>(), ST = NF + 1;
  extern __shared__ float2 zrow[];  // [RB / 2][ST]: one beta pair per complex transform
  __shared__ int s_pos[NF];
  const So3Out o = bt.out[blockIdx.z];
  const int r = blockIdx.y;
  const int k0 = blockIdx.x * RB;
  const int nk = min(RB, n - k0);
  const int np = (nk + 1) >> 1;
  for (int b = threadIdx.x; b < n; b += blockDim.x) s_pos[b] = fixed_freq2pos<NF>(b);
  __syncthreads();
  const int alpha = fixed_pos2freq<NF>(r);
  const float2* __restrict__ Sr = o.S + (size_t)r * Bo * n + k0;
  constexpr int U = 2;  // loads in flight per thread
  for (int e0 = threadIdx.x; e0 < np * Bo; e0 += U * blockDim.x) {
    float4 w[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int e = e0 + u * blockDim.x;
      const int b = e / np, pp = e - b * np;
      const bool ok = e < np * Bo && b < bw_in;
      w[u] = ok ? *reinterpret_cast<const float4*>(Sr + (size_t)b * n + 2 * pp) : make_float4(0.f, 0.f, 0.f, 0.f);
      if (ok && 2 * pp + 1 >= nk) w[u].z = w[u].w = 0.f;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int e = e0 + u * blockDim.x;
      if (e >= np * Bo) continue;
      const int b = e / np, pp = e - b * np;
      const float2 u0 = make_float2(w[u].x, w[u].y), u1 = make_float2(w[u].z, w[u].w);
      float2* z = zrow + pp * ST;
      if (b == 0) {
        z[s_pos[0]] = make_float2(u0.x, u1.x);
        z[s_pos[Bo]] = make_float2(0.f, 0.f);
      } else {
        z[s_pos[b]] = make_float2(u0.x + u1.y, u1.x - u0.y);      // conj(u0) + i conj(u1)
        z[s_pos[n - b]] = make_float2(u0.x - u1.y, u0.y + u1.x);  // u0 + i u1
      }
    }
  }
  __syncthreads();
  fft_tail<NF, true, false, true, kSo3TailThreads>(zrow, np, ST, plan.tw);
  const float K = (float)((1.0 / (double)n) * ((double)Bo / M_PI));
  // per thread: the largest value, the lowest index among equal ones
  float bv = -1.0f;
  uint32_t bi = 0xffffffffu;
  for (int e = threadIdx.x; e < np * n; e += blockDim.x) {
    const int pp = e / n, g = e - pp * n;
    const float2 z = zrow[pp * ST + g];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int j = 2 * pp + h;
      if (j < nk) {
        const float v = (h ? z.y : z.x) * K;
        const float v2 = v * v;
        const uint32_t idx = ((uint32_t)(k0 + j) * n + (uint32_t)alpha) * n + g;
        if (v2 > bv || (v2 == bv && idx < bi)) {
          bv = v2;
          bi = idx;
        }
        if (o.volume) o.volume[idx] = v2;
      }
    }
  }
  warp_argmax_commit(bi == 0xffffffffu ? 0ull : pack_argmax(bv, bi), o.argmax);
}

template <int NF>
static cudaError_t so3_attrs() {
  const int m = 227 * 1024;
  cudaError_t e = cudaFuncSetAttribute(k_so3_fft_a<NF, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, m);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_so3_fft_a<NF, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, m);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_so3_fft_a<NF, 5>, cudaFuncAttributeMaxDynamicSharedMemorySize, m);
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
  if (e == cudaSuccess) e = so3_tc_init_attributes();
  return e;
}

cudaError_t launch_so3_synth(const So3Args& a, cudaStream_t st) {
  if (a.batch.count < 1 || a.batch.count > kMaxWave) return cudaErrorInvalidValue;
  const int ncls = a.bw_in * (a.bw_in + 1) / 2;
  const int n = 2 * a.bw_out;
  int thr = (((n + kSynthBetas - 1) / kSynthBetas + 31) / 32) * 32;
  if (thr > 512) thr = 512;
  const size_t sm1 = (size_t)a.bw_in * 3 * sizeof(double) + 2 * sizeof(double) + (size_t)a.bw_in * 4 * sizeof(float2);
  k_so3_synth<<<dim3(ncls, a.batch.count), thr, sm1, st>>>(a.bw_in, a.bw_out, a.batch, a.beta_tab, a.wig_tab);
  count_launches(1);
  return cudaGetLastError();
}

// The gamma transform: packed pairs on the register-tail engine where the
// length has a tail plan, one sequence per transform otherwise.
template <int NF>
static void launch_so3_c2r(const So3Args& a, int n, cudaStream_t st) {
  if constexpr (Tail<NF>::ok) {
    constexpr int RB = c2r_pair_rows<NF>();
    dim3 g((n + RB - 1) / RB, n, a.batch.count);
    k_so3_c2r_tail<NF><<<g, kSo3TailThreads, (size_t)(RB / 2) * (NF + 1) * sizeof(float2), st>>>(a.bw_in, a.batch,
                                                                                               *a.plan);
  } else {
    dim3 g((n + 15) / 16, n, a.batch.count);
    k_so3_c2r<NF><<<g, 256, (size_t)16 * n * sizeof(float2) + (size_t)n * sizeof(int), st>>>(a.bw_in, a.bw_out,
                                                                                            a.batch, *a.plan);
  }
}

template <int NF>
static void launch_so3_fft_a(const So3Args& a, int n, int wt, cudaStream_t st) {
  dim3 g((n + wt - 1) / wt, a.bw_in, a.batch.count);
  const size_t sm = (size_t)n * wt * sizeof(float2);
  if (wt == 8)
    k_so3_fft_a<NF, 3><<<g, kSo3FftAThreads, sm, st>>>(a.bw_in, a.bw_out, a.batch, *a.plan);
  else if (wt == 32)
    k_so3_fft_a<NF, 5><<<g, kSo3FftAThreads, sm, st>>>(a.bw_in, a.bw_out, a.batch, *a.plan);
  else
    k_so3_fft_a<NF, 4><<<g, kSo3FftAThreads, sm, st>>>(a.bw_in, a.bw_out, a.batch, *a.plan);
}

bool so3_beta_tile_ok(int bw_out, int wt) {
  return (wt == 8 || wt == 16 || wt == 32) && (size_t)2 * bw_out * wt * sizeof(float2) <= 227u * 1024u;
}

cudaError_t launch_so3_fft(const So3Args& a, cudaStream_t st) {
  if (a.batch.count < 1 || a.batch.count > kMaxWave) return cudaErrorInvalidValue;
  const int n = 2 * a.bw_out;
  const int wt = so3_beta_tile_ok(a.bw_out, a.beta_tile) ? a.beta_tile : 16;
  PHGPU_DISPATCH_N(n, launch_so3_fft_a<NF>(a, n, wt, st); launch_so3_c2r<NF>(a, n, st));
  count_launches(2);
  return cudaGetLastError();
}

}  // namespace phgpu
