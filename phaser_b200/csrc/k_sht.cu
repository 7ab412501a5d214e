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
#include <algorithm>

#include "kernels.h"
#include "tc_gemm.cuh"

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

// The transform runs in two kernels over both sides' signals at once.
//
// k_sht_phi: F_m(theta_k) for every signal, order m < B and row k.  Rows are
// real, so rows a and b of a block are transformed together as z = x_a + i x_b
// by one complex FFT (the length's plan; digit-reversed output) and split as
// X_a[m] = (Z[m] + conj Z[-m]) / 2, X_b[m] = (Z[m] - conj Z[-m]) / 2i.
//
// k_sht_leg: block per (order pair {m, B-1-m}, side), so every block carries
// B + 1 Legendre degrees of one side's channels: per order, a product of the
// table rows [degrees x 2B] with the channels' F [2B x channels].  The
// block's slice of the table (the rows of orders m0 and m1, each order
// contiguous) is streamed into shared memory by asynchronous copies -- in one
// piece when it fits, else through two slots, one chunk in flight while the
// other is consumed.  Thread (degree, quarter of the rows k) accumulates every
// channel's real and imaginary part from one table load, two k at a time;
// the four quarters are summed through shared memory.
constexpr int kPhiRows = 8;  // rows per block: kPhiRows / 2 complex transforms
constexpr int kPhiThreads = 128;
constexpr int kLegTasks = 128;  // degrees per round
constexpr int kLegParts = 4;    // threads per degree (quarters of the rows k)
constexpr int kLegThreads = kLegTasks * kLegParts;
constexpr int kMaxSig = 4;  // channels per side
constexpr size_t kShtSmemLimit = (size_t)227 * 1024;

template <int NF>
__global__ void __launch_bounds__(kPhiThreads) k_sht_phi(int bw, int n_data, size_t side_stride,
                                                         const float* __restrict__ sig, FftPlan plan,
                                                         float2* __restrict__ fphi) {
  extern __shared__ float2 zr[];  // [kPhiRows / 2][n] packed row pairs
  const int n = 2 * bw;
  const int s = blockIdx.y, side = s / n_data, c = s - side * n_data;
  const float* S = sig + side * side_stride + (size_t)c * n * n;
  const int k0 = blockIdx.x * kPhiRows;
  const int nr = min(kPhiRows, n - k0);  // even: n and k0 are
  const int np = nr / 2;
  // items of two neighbouring samples of a row pair (8-byte loads: rows are
  // 2B floats), all of a thread's loads in flight together
  const int nh = n / 2;
  constexpr int U = 4;
  for (int i0 = threadIdx.x; i0 < np * nh; i0 += U * blockDim.x) {
    float2 a[U], b[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = i0 + u * blockDim.x;
      const int p = i / nh, j = 2 * (i - p * nh);
      const float* r0 = S + (size_t)(k0 + 2 * p) * n + j;
      const bool ok = i < np * nh;
      a[u] = ok ? __ldg(reinterpret_cast<const float2*>(r0)) : make_float2(0.f, 0.f);
      b[u] = ok ? __ldg(reinterpret_cast<const float2*>(r0 + n)) : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = i0 + u * blockDim.x;
      if (i < np * nh) {
        const int p = i / nh, j = 2 * (i - p * nh);
        zr[p * n + j] = make_float2(a[u].x, b[u].x);
        zr[p * n + j + 1] = make_float2(a[u].y, b[u].y);
      }
    }
  }
  __syncthreads();
  fft_any<NF, false>(zr, np, n, 1, plan);
  const float half = (float)(0.5 * 2.5066282746310002 / (double)n);  // sqrt(2 pi) / 2B, halved
  for (int e = threadIdx.x; e < bw * np; e += blockDim.x) {
    const int m = e / np, p = e - m * np;
    const float2 za = zr[p * n + freq2pos<NF>(m, plan)];
    const float2 zb = zr[p * n + freq2pos<NF>(m == 0 ? 0 : n - m, plan)];
    float2* out = fphi + ((size_t)s * bw + m) * n + k0 + 2 * p;
    out[0] = make_float2((za.x + zb.x) * half, (za.y - zb.y) * half);
    out[1] = make_float2((za.y + zb.y) * half, (zb.x - za.x) * half);
  }
}

__device__ __forceinline__ void cp_async8(float* dst, const float* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}


__global__ void __launch_bounds__(kLegThreads) k_sht_leg(int bw, int n_data, int cr, int nslot,
                                                         const float* __restrict__ table,
                                                         const float2* __restrict__ fphi, float2* __restrict__ coef) {
  extern __shared__ float2 sh[];
  const int n = 2 * bw;
  const int rs = n + 2;  // table row stride in shared memory (8-byte aligned, conflict-free 8-byte reads)
  const int m0 = blockIdx.x, m1 = bw - 1 - blockIdx.x;
  const int nm = (m1 > m0) ? 2 : 1;
  const int side = blockIdx.y;
  float2* f = sh;                                                             // [2][n][kMaxSig]
  float* part = reinterpret_cast<float*>(sh + (size_t)2 * n * kMaxSig);       // [kLegParts][kLegTasks][2 kMaxSig]
  float* ring = part + (size_t)kLegParts * kLegTasks * 2 * kMaxSig;           // [nslot][cr][rs]
  const size_t slot = (size_t)cr * rs;
  // tasks t < nl0: order m0, degree m0 + t; then order m1, degree m1 + t - nl0
  const int nl0 = bw - m0;
  const int ntask = nl0 + (nm == 2 ? bw - m1 : 0);
  const float* seg0 = table + legendre_offset(m0, bw);
  const float* seg1 = table + legendre_offset(m1, bw);
  auto stage_tasks = [&](float* dst, int t0) {
    const int t1 = min(t0 + cr, ntask);
    const int rows = t1 - t0, half = n / 2;
    for (int i = threadIdx.x; i < rows * half; i += blockDim.x) {
      const int r = i / half, j = 2 * (i - r * half);
      const int t = t0 + r;
      const float* src = (t < nl0 ? seg0 + (size_t)t * n : seg1 + (size_t)(t - nl0) * n) + j;
      cp_async8(dst + (size_t)r * rs + j, src);
    }
  };
  stage_tasks(ring, 0);
  cp_async_commit();
  // F rows of both orders, channels innermost: f[(h n + k) kMaxSig + q]
  for (int e = threadIdx.x; e < 2 * n * kMaxSig; e += blockDim.x) {
    const int q = e % kMaxSig, hk = e / kMaxSig, h = hk / n, k = hk - h * n;
    const int m = h ? m1 : m0;
    f[e] = (q < n_data && (h == 0 || nm == 2)) ? fphi[(((size_t)side * n_data + q) * bw + m) * n + k]
                                                : make_float2(0.f, 0.f);
  }
  const int tl = threadIdx.x % kLegTasks, quarter = threadIdx.x / kLegTasks;
  const int kq = ((n / 2 + kLegParts - 1) / kLegParts) * 2;  // rows k per quarter (even)
  const int ka = quarter * kq, kb = min(n, ka + kq);
  const int nc = (ntask + cr - 1) / cr;
  for (int c = 0; c < nc; ++c) {
    if (c + 1 < nc) stage_tasks(ring + ((c + 1) % nslot) * slot, (c + 1) * cr);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const float* chunk = ring + (c % nslot) * slot;
    const int tc = min(cr, ntask - c * cr);  // tasks in this chunk
    for (int r0 = 0; r0 < tc; r0 += kLegTasks) {
      const int r = r0 + tl;
      float acc[2 * kMaxSig];
#pragma unroll
      for (int q = 0; q < 2 * kMaxSig; ++q) acc[q] = 0.f;
      if (r < tc) {
        const int h = c * cr + r < nl0 ? 0 : 1;
        const float* trow = chunk + (size_t)r * rs;
        const float4* fh = reinterpret_cast<const float4*>(f + (size_t)h * n * kMaxSig);
        for (int k = ka; k < kb; k += 2) {
          const float2 t = *reinterpret_cast<const float2*>(trow + k);
#pragma unroll
          for (int q2 = 0; q2 < kMaxSig / 2; ++q2) {
            const float4 x0 = fh[(size_t)k * (kMaxSig / 2) + q2];        // channels 2 q2, 2 q2 + 1 at k
            const float4 x1 = fh[(size_t)(k + 1) * (kMaxSig / 2) + q2];  // at k + 1
            acc[4 * q2 + 0] = fmaf(t.x, x0.x, fmaf(t.y, x1.x, acc[4 * q2 + 0]));
            acc[4 * q2 + 1] = fmaf(t.x, x0.y, fmaf(t.y, x1.y, acc[4 * q2 + 1]));
            acc[4 * q2 + 2] = fmaf(t.x, x0.z, fmaf(t.y, x1.z, acc[4 * q2 + 2]));
            acc[4 * q2 + 3] = fmaf(t.x, x0.w, fmaf(t.y, x1.w, acc[4 * q2 + 3]));
          }
        }
      }
      float* pp = part + ((size_t)quarter * kLegTasks + tl) * 2 * kMaxSig;
#pragma unroll
      for (int q = 0; q < 2 * kMaxSig; ++q) pp[q] = acc[q];
      __syncthreads();
      // sum the quarters: thread (task, value)
      for (int e = threadIdx.x; e < kLegTasks * 2 * kMaxSig; e += blockDim.x) {
        const int rr = e / (2 * kMaxSig), v = e - rr * 2 * kMaxSig, q = v >> 1;
        const int rt = r0 + rr;
        if (rt < tc && q < n_data) {
          float sum = 0.f;
#pragma unroll
          for (int g = 0; g < kLegParts; ++g) sum += part[((size_t)g * kLegTasks + rr) * 2 * kMaxSig + v];
          const int task = c * cr + rt;
          const int h = task < nl0 ? 0 : 1;
          const int m = h ? m1 : m0;
          const int l = m + (h ? task - nl0 : task);
          float* dst = reinterpret_cast<float*>(&coef[(((size_t)side * n_data + q) * bw + l) * bw + m]);
          dst[v & 1] = sum;
        }
      }
      __syncthreads();  // partials and (after the last round) the slot are reused
    }
  }
}

namespace {
// Table rows per chunk and slots: the whole slice of B + 1 rows in one slot
// when it fits beside the F rows, else two slots of as many rows as fit.
bool leg_chunking(int bw, int n_data, int* cr, int* nslot, size_t* smem) {
  (void)n_data;
  const size_t n = 2 * (size_t)bw;
  const size_t fixed = 2 * n * kMaxSig * sizeof(float2) + (size_t)kLegParts * kLegTasks * 2 * kMaxSig * sizeof(float);
  if (fixed >= kShtSmemLimit) return false;
  const size_t row = (n + 2) * sizeof(float);
  const size_t one = (kShtSmemLimit - fixed) / row;
  if (one >= (size_t)bw + 1) {
    *cr = bw + 1;
    *nslot = 1;
  } else {
    *cr = (int)(one / 2);
    *nslot = 2;
  }
  if (*cr < 1) return false;
  *smem = fixed + (size_t)*nslot * *cr * row;
  return true;
}
}  // namespace

size_t sht_scratch_entries(int bw) { return (size_t)2 * kMaxSig * bw * 2 * bw; }

struct LegendreGemm;
template <int PREC>
__global__ void k_sht_leg_tc(TcGemmArgs g, LegendreGemm prob);

cudaError_t sht_init_attributes() {
  cudaError_t e = cudaFuncSetAttribute(k_sht_leg, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kShtSmemLimit);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_sht_leg_tc<kSo3Tf32x3>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_sht_leg_tc<kSo3Bf16x3>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
  return e;
}

cudaError_t launch_sht_phi(const ShtArgs& a, cudaStream_t st) {
  if (a.n_data < 1 || a.n_data > kMaxSig) return cudaErrorInvalidValue;
  const int n = 2 * a.bw;
  if (a.plan->n != n) return cudaErrorInvalidValue;
  dim3 g1((n + kPhiRows - 1) / kPhiRows, 2 * a.n_data);
  const size_t sm1 = (size_t)(kPhiRows / 2) * n * sizeof(float2);
  PHGPU_DISPATCH_N(n, k_sht_phi<NF><<<g1, kPhiThreads, sm1, st>>>(a.bw, a.n_data, a.side_stride, a.signal,
                                                                   *a.plan, a.fphi));
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_sht(const ShtArgs& a, cudaStream_t st) {
  int cr = 0, nslot = 0;
  size_t sm = 0;
  if (a.n_data < 1 || a.n_data > kMaxSig || !leg_chunking(a.bw, a.n_data, &cr, &nslot, &sm))
    return cudaErrorInvalidValue;
  cudaError_t e = launch_sht_phi(a, st);
  if (e != cudaSuccess) return e;
  if (a.table_tc) {
    ShtBatch b;
    b.count = 1;
    b.fphi[0] = a.fphi;
    b.coef[0] = a.coef;
    return launch_sht_leg_tc(a.bw, a.n_data, b, a.table_tc, a.precision, a.tc_chunk, a.status, st);
  }
  dim3 g2((a.bw + 1) / 2, 2);
  k_sht_leg<<<g2, kLegThreads, sm, st>>>(a.bw, a.n_data, cr, nslot, a.table, a.fphi, a.coef);
  count_launches(1);
  return cudaGetLastError();
}

// ------------------------------------------------------------------ tensor-core Legendre contraction
//
// fhat(l, m) = sum_k T[m][l][k] F_m(theta_k) for every signal as a tc_gemm
// problem (tc_gemm.cuh): class = order m (largest first), rows = degrees
// l = m .. B-1, k = the 2B rows theta_k, one group of 8 columns per (request,
// side): the four channels' real and imaginary parts.  A wave of K requests
// reads the table once.  Table layout per order: [k / 4][B - m][4] floats,
// k padded to a multiple of 8 with zeros (legendre_tc_offset), followed by the
// B row sums S_l = sum_k T[0][l][k] (FP64 sums of the FP32 table).
//
// Order 0 contracts F_0(theta_k) - D with D = F_0(theta_B) (the ring below the
// equator) and adds D S_l afterwards: the same sum, but a range or intensity
// channel's large constant part no longer enters the tensor-core accumulation,
// whose truncation error scales with the magnitude of the partial sums.

__host__ __device__ inline int legendre_tc_kdim(int bw) { return (2 * bw + 7) & ~7; }

__host__ __device__ inline size_t legendre_tc_offset(int m, int bw) {
  return (size_t)legendre_tc_kdim(bw) * ((size_t)m * bw - (size_t)m * (m - 1) / 2);
}

size_t legendre_tc_floats(int bw) { return legendre_tc_offset(bw, bw) + (size_t)bw; }

// T_tc from the row-major table T[m][l][k] (k fastest): one thread per entry.
__global__ void k_legendre_tc_layout(int bw, const float* __restrict__ T, float* __restrict__ Ttc) {
  const int n = 2 * bw, kd = legendre_tc_kdim(bw);
  const int m = blockIdx.y;
  const int rows = bw - m;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < rows * kd; e += gridDim.x * blockDim.x) {
    const int r = e / kd, k = e - r * kd;
    const float v = k < n ? T[legendre_offset(m, bw) + (size_t)r * n + k] : 0.0f;
    Ttc[legendre_tc_offset(m, bw) + ((size_t)(k >> 2) * rows + r) * 4 + (k & 3)] = v;
  }
}

// S_l = sum_k T[0][l][k] in FP64, one thread per degree.
__global__ void k_legendre_row_sums(int bw, const float* __restrict__ T, float* __restrict__ S) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= bw) return;
  const int n = 2 * bw;
  const float* row = T + legendre_offset(0, bw) + (size_t)l * n;
  double s = 0.0;
  for (int k = 0; k < n; ++k) s += (double)row[k];
  S[l] = (float)s;
}

cudaError_t launch_legendre_tc_layout(int bw, const float* table, float* table_tc, cudaStream_t st) {
  k_legendre_tc_layout<<<dim3(64, bw), 256, 0, st>>>(bw, table, table_tc);
  k_legendre_row_sums<<<(bw + 127) / 128, 128, 0, st>>>(bw, table, table_tc + legendre_tc_offset(bw, bw));
  count_launches(2);
  return cudaGetLastError();
}

struct LegendreGemm {
  int bw, n_data;
  const float* table;
  ShtBatch b;

  __device__ int classes() const { return bw; }
  __device__ TcClass cls(int m) const {
    TcClass t;
    t.rows = bw - m;
    t.kdim = legendre_tc_kdim(bw);
    t.a = table + legendre_tc_offset(m, bw);
    t.u0 = m;
    t.u1 = 0;
    return t;
  }
  __device__ void bvals(const TcClass& c, int grp, int k, float v[8]) const {
    const int r = grp >> 1, side = grp & 1, n = 2 * bw;
#pragma unroll
    for (int q = 0; q < kMaxSig; ++q) {
      float2 f = make_float2(0.f, 0.f);
      if (q < n_data && k < n) {
        const float2* F = b.fphi[r] + (((size_t)side * n_data + q) * bw + c.u0) * n;
        f = __ldg(&F[k]);
        if (c.u0 == 0) {
          const float2 d = __ldg(&F[bw]);
          f = make_float2(f.x - d.x, f.y - d.y);
        }
      }
      v[2 * q] = f.x;
      v[2 * q + 1] = f.y;
    }
  }
  __device__ void store(const TcClass& c, int grp, int row, const float v[8]) const {
    const int r = grp >> 1, side = grp & 1, l = c.u0 + row, n = 2 * bw;
    for (int q = 0; q < n_data; ++q) {
      float2 o = make_float2(v[2 * q], v[2 * q + 1]);
      if (c.u0 == 0) {
        const float2 d = __ldg(&b.fphi[r][(((size_t)side * n_data + q) * bw) * n + bw]);
        const float sl = __ldg(&table[legendre_tc_offset(bw, bw) + l]);
        o = make_float2(fmaf(d.x, sl, o.x), fmaf(d.y, sl, o.y));
      }
      b.coef[r][(((size_t)side * n_data + q) * bw + l) * bw + c.u0] = o;
    }
  }
};

template <int PREC>
__global__ void __launch_bounds__(kTcThreads, kTcCtasPerSm) k_sht_leg_tc(TcGemmArgs g, LegendreGemm prob) {
  tc_class_gemm<PREC>(g, prob);
}

bool sht_leg_tc_supported(int bw, int count, int precision) {
  TcGemmArgs g;
  return count >= 1 && count <= kMaxWave && tc_gemm_geom(bw, 2 * count, precision, 0, true, &g);
}

cudaError_t launch_sht_leg_tc(int bw, int n_data, const ShtBatch& b, const float* table_tc, int precision,
                              int chunk, unsigned long long* status, cudaStream_t st) {
  if (n_data < 1 || n_data > kMaxSig || b.count < 1 || b.count > kMaxWave) return cudaErrorInvalidValue;
  TcGemmArgs g;
  if (!tc_gemm_geom(bw, 2 * b.count, precision, chunk, true, &g) &&
      !tc_gemm_geom(bw, 2 * b.count, precision, 0, true, &g))
    return cudaErrorInvalidValue;
  g.status = status;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  LegendreGemm prob;
  prob.bw = bw;
  prob.n_data = n_data;
  prob.table = table_tc;
  prob.b = b;
  const int grid = bw < sms * g.ctas_per_sm ? bw : sms * g.ctas_per_sm;
  if (precision == kSo3Tf32x3)
    k_sht_leg_tc<kSo3Tf32x3><<<grid, kTcThreads, g.smem, st>>>(g, prob);
  else
    k_sht_leg_tc<kSo3Bf16x3><<<grid, kTcThreads, g.smem, st>>>(g, prob);
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

// One thread per (l, m) with |m| <= l; both sides; request blockIdx.y.
__global__ void k_fuse_s2(FuseS2Args a) {
  const int bw = a.bw;
  const float2* __restrict__ coef = a.coef_b[blockIdx.y];
  float2* __restrict__ fused = a.fused_b[blockIdx.y];
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
    const float2* base = coef + (size_t)side * a.n_data_ch * bw * bw;
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
    fused[((size_t)side * bw + l) * w + mi] = r;
  }
}

// SphRegistration's single signal (SphericalCorrelation::retrieveInterpolation,
// phaser_core/src/backend/correlation/spherical-correlation.cc:103-112):
// 0.6 * intensity + 0.4 * range of every direction, in double, for both
// sides; samples [side][c][n] with channels {range, intensity, ...}.
__global__ void k_mix_signal(const float* __restrict__ samples, size_t side_stride, int n, float* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 2 * n) return;
  const int side = i / n, k = i - side * n;
  const float* s = samples + (size_t)side * side_stride;
  out[i] = (float)__dadd_rn(__dmul_rn(0.6, (double)s[n + k]), __dmul_rn(0.4, (double)s[k]));
}

cudaError_t launch_mix_signal(const float* samples, size_t side_stride, int n, float* out, cudaStream_t st) {
  k_mix_signal<<<(2 * n + 255) / 256, 256, 0, st>>>(samples, side_stride, n, out);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_fuse_s2(const FuseS2Args& a0, cudaStream_t st) {
  FuseS2Args a = a0;
  if (a.count < 1) {
    a.count = 1;
    a.coef_b[0] = a.coef;
    a.fused_b[0] = a.fused;
  }
  if (a.count > kMaxWave) return cudaErrorInvalidValue;
  const int tot = a.bw * (2 * a.bw - 1);
  k_fuse_s2<<<dim3((tot + 255) / 256, a.count), 256, 0, st>>>(a);
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace phgpu
