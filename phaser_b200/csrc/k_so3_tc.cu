// Wigner-d table and tensor-core SO(3) synthesis (sm_100a tcgen05).
//
// Reference behaviour: the sum S_{m1 m2}(beta_k) = sum_l c(l, m1, m2)
// dtilde^l_{m1 m2}(beta_k) of SOFT's wigNaiveSynthesis_fftw
// (phaser_core/lib/SOFT/wignerTransforms_fftw.c:407-442), with the d-values
// SOFT regenerates per call by genWigTrans_L2 / wigSpec_L2
// (makeWigner.c:324-387,634-698) and the coefficient product of
// so3CombineCoef_fftw (so3_correlate_fftw.c:102-161).
//
// Table (k_so3_table, once per context): for every order class (p, q),
// 0 <= p <= q < B, the L2-normalised d^{q+i}_{pq}(beta_k), i < B - q, k < 2 bw_out,
// from the FP64 three-term recurrence, rounded once to FP32.  A class feeds
// four (m1, m2) outputs through the d-symmetries (so3_common.cuh), so the
// table holds one eighth of the (m1, m2) plane.  Block layout per class:
// [degree group of 4][beta][4] floats (16 bytes = one row of an 8 x 16-byte
// core matrix of the tensor-core operand), degrees padded to 8 with zeros.
//
// Synthesis (k_so3_synth_tc): per class a GEMM (tc_gemm.cuh)
//   Out[beta][j] = sum_i D[beta][i] C[j][i],
// j = 8 r + 2 v + {re, im} for request r of the wave and output v of the class,
// so a wave of K requests reads the table once; the coefficient operand is
// formed per chunk from the fused spectra, the epilogue writes the four
// outputs of every request into S[a][b][beta] (coalesced along beta).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <vector>

#include "kernels.h"
#include "so3_common.cuh"
#include "tc_gemm.cuh"

namespace phgpu {

bool so3_tc_supported(int bw_out, int count, int precision, int chunk) {
  TcGemmArgs g;
  return bw_out <= 256 && count >= 1 && count <= kMaxWave &&
         tc_gemm_geom(2 * bw_out, count, precision, chunk, false, &g);
}

size_t so3_table_layout(int bw_in, int bw_out, std::vector<size_t>* off) {
  const int n = 2 * bw_out;
  const int ncls = bw_in * (bw_in + 1) / 2;
  off->resize(ncls);
  size_t o = 0;
  for (int c = 0; c < ncls; ++c) {
    int p, q;
    so3_class(c, &p, &q);
    const int nlp = ((bw_in - q) + 7) & ~7;
    (*off)[c] = o;
    o += (size_t)nlp * n;
  }
  return o;
}

// ------------------------------------------------------------------ table

__global__ void k_so3_table(int bw_in, int bw_out, const double* __restrict__ btab, const double* __restrict__ wtab,
                            const size_t* __restrict__ class_off, float* __restrict__ table) {
  extern __shared__ double sm[];
  double* fa = sm;
  double* fb = fa + bw_in;
  double* gs = fb + bw_in;
  int p, q;
  so3_class(blockIdx.x, &p, &q);
  const int nl = bw_in - q;
  const int nlp = (nl + 7) & ~7;
  const WigTab W = wig_tab(wtab, bw_in);
  const int b1 = bw_in + 1;
  for (int i = threadIdx.x; i < nl; i += blockDim.x) wig_factors(W, b1, p, q, q + i, &fa[i], &fb[i], &gs[i]);
  __syncthreads();
  const double lnorm = wig_lnorm(W, p, q);
  const int n = 2 * bw_out;
  float* __restrict__ T = table + class_off[blockIdx.x];
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    const double cb = __ldg(&btab[k]);
    double dcur = wig_seed(btab, n, k, lnorm, p, q), dprev = 0.0;
    for (int i = 0; i < nlp; ++i) {
      T[(size_t)(i >> 2) * n * 4 + (size_t)k * 4 + (i & 3)] = i < nl ? (float)dcur : 0.0f;
      if (i < nl) {
        const double dn = wig_step(fa[i], fb[i], gs[i], cb, dprev, dcur);
        dprev = dcur;
        dcur = dn;
      }
    }
  }
}

cudaError_t launch_so3_table(int bw_in, int bw_out, const double* beta_tab, const double* wig_tab,
                             const size_t* class_off, float* table, cudaStream_t st) {
  const int ncls = bw_in * (bw_in + 1) / 2;
  const int thr = 2 * bw_out >= 256 ? 256 : 128;
  k_so3_table<<<ncls, thr, (size_t)3 * bw_in * sizeof(double), st>>>(bw_in, bw_out, beta_tab, wig_tab, class_off,
                                                                    table);
  count_launches(1);
  return cudaGetLastError();
}

// ------------------------------------------------------------------ synthesis

// The Wigner synthesis as a tc_gemm problem: class c = order pair (p, q),
// rows = betas, k = degrees q + i, one group of 8 columns per request.
struct WignerGemm {
  int bw_in, n;
  const float* table;
  const size_t* class_off;
  const double* wtab;
  So3Batch bt;

  __device__ int classes() const { return bw_in * (bw_in + 1) / 2; }
  __device__ TcClass cls(int c) const {
    int p, q;
    so3_class(c, &p, &q);
    TcClass t;
    t.rows = n;
    t.kdim = ((bw_in - q) + 7) & ~7;
    t.a = table + class_off[c];
    t.u0 = p;
    t.u1 = q;
    return t;
  }
  __device__ void bvals(const TcClass& c, int r, int i, float v[8]) const {
    const int p = c.u0, q = c.u1;
    if (i < bw_in - q) {
      const WigTab W = wig_tab(wtab, bw_in);
      const int l = q + i;
      float2 cv[4];
      so3_coefs(bt.fused[r], bw_in, p, q, l, (float)__ldg(&W.wl[l]), cv);
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        v[2 * u] = cv[u].x;
        v[2 * u + 1] = cv[u].y;
      }
    } else {
#pragma unroll
      for (int u = 0; u < 8; ++u) v[u] = 0.0f;
    }
  }
  __device__ void store(const TcClass& c, int r, int k, const float v[8]) const {
    float2 acc[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) acc[u] = make_float2(v[2 * u], v[2 * u + 1]);
    so3_store(bt.out[r].S, n, c.u0, c.u1, k, acc);
  }
};

template <int PREC>
__global__ void __launch_bounds__(kTcThreads, kTcCtasPerSm) k_so3_synth_tc(TcGemmArgs g, WignerGemm prob) {
  tc_class_gemm<PREC>(g, prob);
}

cudaError_t so3_tc_init_attributes() {
  cudaError_t e = cudaFuncSetAttribute(k_so3_synth_tc<kSo3Tf32x3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       227 * 1024);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_so3_synth_tc<kSo3Bf16x3>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
  return e;
}

cudaError_t launch_so3_synth_tc(const So3Args& a, const So3Table& t, unsigned long long* status, cudaStream_t st) {
  TcGemmArgs g;
  if (a.bw_out > 256 || a.batch.count < 1 || a.batch.count > kMaxWave) return cudaErrorInvalidValue;
  if (!tc_gemm_geom(2 * a.bw_out, a.batch.count, t.precision, a.tc_chunk, false, &g) &&
      !tc_gemm_geom(2 * a.bw_out, a.batch.count, t.precision, 0, false, &g))
    return cudaErrorInvalidValue;
  g.status = status;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  WignerGemm prob;
  prob.bw_in = a.bw_in;
  prob.n = 2 * a.bw_out;
  prob.table = t.table;
  prob.class_off = t.class_off;
  prob.wtab = a.wig_tab;
  prob.bt = a.batch;
  const int ncls = a.bw_in * (a.bw_in + 1) / 2;
  const int grid = ncls < sms * g.ctas_per_sm ? ncls : sms * g.ctas_per_sm;
  if (t.precision == kSo3Tf32x3)
    k_so3_synth_tc<kSo3Tf32x3><<<grid, kTcThreads, g.smem, st>>>(g, prob);
  else
    k_so3_synth_tc<kSo3Bf16x3><<<grid, kTcThreads, g.smem, st>>>(g, prob);
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace phgpu
