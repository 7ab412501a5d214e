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
// Synthesis (k_so3_synth_tc): per class a GEMM
//   Out[beta][j] = sum_i D[beta][i] C[j][i],
// j = 8 r + 2 v + {re, im} for request r of the wave and output v of the class,
// so a wave of K requests reads the table once.  Both operands are split
// into a high and a low part and multiplied as hi*hi + hi*lo + lo*hi with FP32
// accumulation in tensor memory:
//   tf32x3: hi = x with the low 13 mantissa bits cleared, lo = x - hi (exact);
//           kind::tf32, relative error of a product ~2^-20;
//   bf16x3: hi = bf16(x), lo = bf16(x - hi); kind::f16 with BF16 inputs,
//           relative error of a product ~2^-17.
// One CTA (256 threads) per SM walks the classes (largest first, round robin).
// Per chunk of KC degrees: one thread issues bulk copies of the table chunk
// into shared memory (mbarrier with a bounded wait), all threads form the
// coefficient operand from the fused spectra and split both operands, one
// thread issues the MMAs (M = 128 rows of betas per tile, N = 8 per request)
// and commits them to an mbarrier; two stages alternate so copies and operand
// preparation overlap the previous chunk's MMAs.  The epilogue reads the
// accumulators with tcgen05.ld (one beta per thread) and writes the four
// outputs of every request into S[a][b][beta] (coalesced along beta).
//
// Operand layout (no swizzle, K-major): element (row, k) at
// (k / kc) * LBO + (row / 8) * 128 + (row % 8) * 16 + (k % kc) * size, with
// kc = 16 bytes / element size, LBO = rows * 16, SBO = 128.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <vector>

#include "kernels.h"
#include "so3_common.cuh"

namespace phgpu {

constexpr int kTcThreads = 256;
constexpr int kTcStages = 2;

struct TcGeom {
  int n;           // betas (2 bw_out)
  int MP;          // rows padded to whole 128-row tiles
  int nmt;         // 128-row tiles
  int N;           // coefficient columns: 8 per request, padded to 16
  int KC;          // degrees per chunk
  int precision;   // kSo3Tf32x3 / kSo3Bf16x3
  uint32_t a32;    // FP32 table chunk: KC * MP * 4 bytes
  uint32_t aconv;  // tf32: low parts (a32); bf16: high + low parts (a32)
  uint32_t bop;    // coefficient operand, high + low
  uint32_t stage;
  uint32_t smem;
  uint32_t tcols;  // tensor-memory columns allocated
};

static bool tc_geom(int bw_out, int count, int precision, TcGeom* g, int chunk = 0) {
  if (precision != kSo3Tf32x3 && precision != kSo3Bf16x3) return false;
  if (count < 1 || count > kMaxWave || bw_out < 1 || bw_out > 256) return false;
  g->precision = precision;
  g->n = 2 * bw_out;
  g->nmt = (g->n + 127) / 128;
  g->MP = g->nmt * 128;
  g->N = ((8 * count + 15) / 16) * 16;
  if (g->nmt * g->N > 512) return false;
  const uint32_t ctrl = 1024;
  for (int KC : {32, 16}) {
    if (chunk && KC != chunk) continue;
    g->KC = KC;
    g->a32 = (uint32_t)KC * g->MP * 4;
    g->aconv = g->a32;
    g->bop = (uint32_t)(precision == kSo3Tf32x3 ? 8 : 4) * KC * g->N;
    g->stage = g->a32 + g->aconv + g->bop;
    g->smem = kTcStages * g->stage + ctrl;
    if (g->smem <= 227u * 1024u) break;
  }
  if (g->smem > 227u * 1024u || (chunk && g->KC != chunk)) return false;
  // at most one CTA per SM, so the tensor-memory allocation never waits
  if (g->smem < 116u * 1024u) g->smem = 116u * 1024u;
  uint32_t c = 32;
  while (c < (uint32_t)(g->nmt * g->N)) c <<= 1;
  g->tcols = c;
  return true;
}

bool so3_tc_supported(int bw_out, int count, int precision, int chunk) {
  TcGeom g;
  return tc_geom(bw_out, count, precision, &g, chunk);
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

// ------------------------------------------------------------------ tcgen05 helpers

__device__ __forceinline__ uint32_t sm_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: start, leading (K) and stride (M/N) byte
// offsets, descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor: FP32 accumulator, A/B format (tf32 = 2, bf16 = 1),
// both K-major, N and M = 128.
__host__ __device__ constexpr uint32_t umma_idesc(uint32_t fmt, uint32_t N) {
  return (1u << 4) | (fmt << 7) | (fmt << 10) | ((N >> 3) << 17) | ((128u >> 4) << 24);
}

template <int PREC>
__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
  if constexpr (PREC == kSo3Tf32x3) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
  } else {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
  }
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Polls an mbarrier phase; gives up after about one second (or at once when
// another thread gave up) and returns false.
__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag, bool honour_abort) {
  uint64_t t0 = 0;
  for (uint32_t it = 0;; ++it) {
    uint32_t ok;
    asm volatile("{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
                 : "=r"(ok)
                 : "r"(bar), "r"(parity)
                 : "memory");
    if (ok) return true;
    if (honour_abort && *abort_flag) return false;
    if ((it & 31u) == 31u) {
      uint64_t now;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
      if (t0 == 0) {
        t0 = now;
      } else if (now - t0 > 1000000000ull) {
        *abort_flag = 1;
        return false;
      }
    }
  }
}

__device__ __forceinline__ uint32_t tf32_hi(uint32_t x) { return x & 0xFFFFE000u; }

// ------------------------------------------------------------------ synthesis

struct TcArgs {
  int bw_in, n, MP, nmt, N, KC, count;
  uint32_t a32, aconv, bop, stage, tcols;
  const float* table;
  const size_t* class_off;
  const double* wtab;
  unsigned long long* status;
};

template <int PREC>
__global__ void __launch_bounds__(kTcThreads, 1) k_so3_synth_tc(TcArgs g, So3Batch bt) {
  extern __shared__ __align__(1024) uint8_t smem[];
  constexpr int ESZ = PREC == kSo3Tf32x3 ? 4 : 2;  // operand element bytes
  constexpr int KCE = 16 / ESZ;                     // elements per 16-byte core row
  constexpr int KSTEP = 32 / ESZ;                   // elements per MMA (two core columns)
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kTcStages * g.stage);  // [load 0, load 1, mma 0, mma 1]
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(bars + 4);
  volatile int* s_abort = reinterpret_cast<volatile int*>(s_tmem + 1);
  // [2 loads, 2 mmas]: 1 + parity of a phase that was issued and may not have been waited for, 0 = none
  int* s_pending = const_cast<int*>(s_abort) + 1;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int n = g.n, MP = g.MP, N = g.N, KC = g.KC;
  const uint32_t lboA = (uint32_t)MP * 16, lboB = (uint32_t)N * 16;

  // zero every operand buffer once: padding rows and columns stay zero
  for (uint32_t e = tid; e < kTcStages * g.stage / 16; e += kTcThreads)
    reinterpret_cast<uint4*>(smem)[e] = make_uint4(0u, 0u, 0u, 0u);
  if (tid == 0) {
    for (int b = 0; b < 4; ++b) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sm_addr(&bars[b])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    *s_abort = 0;
    for (int b = 0; b < 4; ++b) s_pending[b] = 0;
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sm_addr(s_tmem)),
                 "r"(g.tcols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;
  const uint32_t idesc = umma_idesc(PREC == kSo3Tf32x3 ? 2u : 1u, (uint32_t)N);
  const WigTab W = wig_tab(g.wtab, g.bw_in);
  const int ncls = g.bw_in * (g.bw_in + 1) / 2;

  uint32_t it = 0;  // chunks processed by this CTA (stage = it & 1)
  for (int c = blockIdx.x; c < ncls; c += gridDim.x) {
    int p, q;
    so3_class(c, &p, &q);
    const int nl = g.bw_in - q;
    const int nlp = (nl + 7) & ~7;
    const int nch = (nlp + KC - 1) / KC;
    const float* __restrict__ Tc = g.table + g.class_off[c];
    for (int ch = 0; ch < nch; ++ch, ++it) {
      const int s = it & 1;
      uint8_t* stage = smem + s * g.stage;
      float* A32 = reinterpret_cast<float*>(stage);
      uint8_t* AX = stage + g.a32;
      uint8_t* BH = stage + g.a32 + g.aconv;
      uint8_t* BL = BH + g.bop / 2;
      const int kcc = min(KC, nlp - ch * KC) / 4;              // 16-byte degree groups of this chunk
      const int ksteps = (kcc * 4 + KSTEP - 1) / KSTEP;        // MMAs along the degrees
      const int kread = ksteps * KSTEP;                        // degrees the MMAs read
      // stage s was last read by the MMAs of chunk it - 2
      if (it >= 2) tc_wait(sm_addr(&bars[2 + s]), ((it >> 1) - 1) & 1, s_abort, true);
      if (tid == 0) s_pending[2 + s] = 0;
      if (tid == 0 && !*s_abort) {
        const uint32_t bytes = (uint32_t)kcc * n * 16;
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sm_addr(&bars[s])), "r"(bytes)
                     : "memory");
        for (int cc = 0; cc < kcc; ++cc) {
          const float* src = Tc + ((size_t)(ch * KC / 4 + cc) * n) * 4;
          asm volatile(
              "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                  sm_addr(A32 + (size_t)cc * MP * 4)),
              "l"(src), "r"((uint32_t)n * 16), "r"(sm_addr(&bars[s]))
              : "memory");
        }
        s_pending[s] = 1 + (int)((it >> 1) & 1);
      }
      // coefficient operand: rows j = 8 r + 2 v + {re, im}, degrees of the chunk
      const int l0 = q + ch * KC;
      for (int e = tid; e < g.count * kread; e += kTcThreads) {
        const int r = e / kread, il = e - r * kread;
        const int l = l0 + il;
        float vals[8];
        if (ch * KC + il < nl) {
          float2 v[4];
          so3_coefs(bt.fused[r], g.bw_in, p, q, l, (float)__ldg(&W.wl[l]), v);
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            vals[2 * u] = v[u].x;
            vals[2 * u + 1] = v[u].y;
          }
        } else {
#pragma unroll
          for (int u = 0; u < 8; ++u) vals[u] = 0.0f;
        }
        const uint32_t off = (uint32_t)(il / KCE) * lboB + (uint32_t)(il % KCE) * ESZ;
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const uint32_t o = off + (uint32_t)(8 * r + u) * 16;
          if constexpr (PREC == kSo3Tf32x3) {
            const uint32_t x = __float_as_uint(vals[u]);
            const uint32_t hi = tf32_hi(x);
            *reinterpret_cast<uint32_t*>(BH + o) = hi;
            *reinterpret_cast<float*>(BL + o) = vals[u] - __uint_as_float(hi);
          } else {
            const __nv_bfloat16 hi = __float2bfloat16_rn(vals[u]);
            *reinterpret_cast<__nv_bfloat16*>(BH + o) = hi;
            *reinterpret_cast<__nv_bfloat16*>(BL + o) = __float2bfloat16_rn(vals[u] - __bfloat162float(hi));
          }
        }
      }
      tc_wait(sm_addr(&bars[s]), (it >> 1) & 1, s_abort, true);
      if (tid == 0) s_pending[s] = 0;
      // split the table chunk
      if constexpr (PREC == kSo3Tf32x3) {
        uint4* hi = reinterpret_cast<uint4*>(A32);
        float4* lo = reinterpret_cast<float4*>(AX);
        for (int e = tid; e < kcc * n; e += kTcThreads) {
          const int cc = e / n, row = e - cc * n;
          const size_t idx = (size_t)cc * MP + row;
          const uint4 x = hi[idx];
          const uint4 h = make_uint4(tf32_hi(x.x), tf32_hi(x.y), tf32_hi(x.z), tf32_hi(x.w));
          hi[idx] = h;
          lo[idx] = make_float4(__uint_as_float(x.x) - __uint_as_float(h.x), __uint_as_float(x.y) - __uint_as_float(h.y),
                                __uint_as_float(x.z) - __uint_as_float(h.z), __uint_as_float(x.w) - __uint_as_float(h.w));
        }
      } else {
        uint4* hi16 = reinterpret_cast<uint4*>(AX);
        uint4* lo16 = reinterpret_cast<uint4*>(AX + g.aconv / 2);
        const float4* src = reinterpret_cast<const float4*>(A32);
        for (int e = tid; e < (kread / 8) * n; e += kTcThreads) {
          const int c16 = e / n, row = e - c16 * n;
          float x[8];
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int cc = 2 * c16 + h;
            const float4 v = cc < kcc ? src[(size_t)cc * MP + row] : make_float4(0.f, 0.f, 0.f, 0.f);
            x[4 * h] = v.x;
            x[4 * h + 1] = v.y;
            x[4 * h + 2] = v.z;
            x[4 * h + 3] = v.w;
          }
          __nv_bfloat162 h2[4], l2[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const __nv_bfloat16 a = __float2bfloat16_rn(x[2 * u]), b = __float2bfloat16_rn(x[2 * u + 1]);
            h2[u] = __halves2bfloat162(a, b);
            l2[u] = __halves2bfloat162(__float2bfloat16_rn(x[2 * u] - __bfloat162float(a)),
                                       __float2bfloat16_rn(x[2 * u + 1] - __bfloat162float(b)));
          }
          hi16[(size_t)c16 * MP + row] = *reinterpret_cast<uint4*>(h2);
          lo16[(size_t)c16 * MP + row] = *reinterpret_cast<uint4*>(l2);
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      if (tid == 0 && !*s_abort) {
        tc_fence_after();
        const uint32_t aH = PREC == kSo3Tf32x3 ? sm_addr(A32) : sm_addr(AX);
        const uint32_t aL = PREC == kSo3Tf32x3 ? sm_addr(AX) : sm_addr(AX + g.aconv / 2);
        const uint32_t bH = sm_addr(BH), bL = sm_addr(BL);
        for (int ks = 0; ks < ksteps; ++ks) {
          for (int t = 0; t < g.nmt; ++t) {
            const uint32_t dt = tmem + (uint32_t)(t * N);
            const uint32_t ao = (uint32_t)ks * 2u * lboA + (uint32_t)t * 2048u;
            const uint32_t bo = (uint32_t)ks * 2u * lboB;
            const uint32_t first = (ch == 0 && ks == 0) ? 0u : 1u;
            umma<PREC>(dt, umma_desc(aH + ao, lboA, 128), umma_desc(bH + bo, lboB, 128), idesc, first);
            umma<PREC>(dt, umma_desc(aH + ao, lboA, 128), umma_desc(bL + bo, lboB, 128), idesc, 1u);
            umma<PREC>(dt, umma_desc(aL + ao, lboA, 128), umma_desc(bH + bo, lboB, 128), idesc, 1u);
          }
        }
        umma_commit(sm_addr(&bars[2 + s]));
        s_pending[2 + s] = 1 + (int)((it >> 1) & 1);
      }
    }
    // epilogue: the last chunk's MMAs complete every accumulation of the class
    const uint32_t last = it - 1;
    tc_wait(sm_addr(&bars[2 + (last & 1)]), (last >> 1) & 1, s_abort, true);
    tc_fence_after();
    const int qd = warp & 3;
    for (int t = warp >> 2; t < g.nmt; t += 2) {
      const int k = t * 128 + qd * 32 + lane;
      for (int r = 0; r < g.count; ++r) {
        uint32_t v[8];
        const uint32_t ta = tmem + ((uint32_t)(qd * 32) << 16) + (uint32_t)(t * N + 8 * r);
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                     : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                     : "r"(ta));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (k < n && !*s_abort) {
          float2 acc[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) acc[u] = make_float2(__uint_as_float(v[2 * u]), __uint_as_float(v[2 * u + 1]));
          so3_store(bt.out[r].S, n, p, q, k, acc);
        }
      }
    }
    tc_fence_before();
    __syncthreads();
  }
  // leave nothing in flight, then release the tensor memory
  if (tid == 0) {
    for (int b = 0; b < 4; ++b)
      if (s_pending[b]) tc_wait(sm_addr(&bars[b]), (uint32_t)(s_pending[b] - 1), s_abort, false);
    if (*s_abort) atomicOr(g.status, 2ull);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(g.tcols) : "memory");
}

cudaError_t so3_tc_init_attributes() {
  cudaError_t e = cudaFuncSetAttribute(k_so3_synth_tc<kSo3Tf32x3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       227 * 1024);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_so3_synth_tc<kSo3Bf16x3>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
  return e;
}

cudaError_t launch_so3_synth_tc(const So3Args& a, const So3Table& t, unsigned long long* status, cudaStream_t st) {
  TcGeom geo;
  if (!tc_geom(a.bw_out, a.batch.count, t.precision, &geo, a.tc_chunk) &&
      !tc_geom(a.bw_out, a.batch.count, t.precision, &geo))
    return cudaErrorInvalidValue;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int ncls = a.bw_in * (a.bw_in + 1) / 2;
  TcArgs g;
  g.bw_in = a.bw_in;
  g.n = geo.n;
  g.MP = geo.MP;
  g.nmt = geo.nmt;
  g.N = geo.N;
  g.KC = geo.KC;
  g.count = a.batch.count;
  g.a32 = geo.a32;
  g.aconv = geo.aconv;
  g.bop = geo.bop;
  g.stage = geo.stage;
  g.tcols = geo.tcols;
  g.table = t.table;
  g.class_off = t.class_off;
  g.wtab = a.wig_tab;
  g.status = status;
  const int grid = ncls < sms ? ncls : sms;
  if (t.precision == kSo3Tf32x3)
    k_so3_synth_tc<kSo3Tf32x3><<<grid, kTcThreads, geo.smem, st>>>(g, a.batch);
  else
    k_so3_synth_tc<kSo3Bf16x3><<<grid, kTcThreads, geo.smem, st>>>(g, a.batch);
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace phgpu
