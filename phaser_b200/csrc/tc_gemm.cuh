// Tensor-core (tcgen05) GEMMs of many small independent classes, with both
// operands split into high and low parts for FP32-level accuracy.
//
// Used by the SO(3) synthesis (k_so3_tc.cu: one class per Wigner order pair
// (p, q)) and the Legendre contraction of the forward SHT (k_sht.cu: one class
// per order m).  For every class c:
//   Out[row][j] = sum_k A_c[row][k] * Bop_c[j][k],   row < rows_c, j < N, k < kdim_c
// where A_c is a stored FP32 table block laid out [k / 4][rows_c][4] (16-byte
// groups of four k per row: the rows of the operand's 8 x 16-byte core
// matrices), and Bop_c is generated per chunk by the problem (8 columns per
// group: a request's four complex values, or a signal pair's channels).
//
// Split products, FP32 accumulation in tensor memory:
//   tf32x3: hi = tf32_rn(x), lo = tf32_rn(x - hi); kind::tf32
//   bf16x3: hi = bf16(x), lo = bf16(x - hi); kind::f16 with BF16 inputs
//   Out = (sum Ahi Bhi) + (sum Ahi Blo + Alo Bhi)
// With `sep` (the Legendre contraction) the two sums accumulate in separate
// tensor-memory columns and are added in FP32 by the epilogue; without it
// (the Wigner-d synthesis, whose wave-wide accumulators would otherwise halve
// the CTAs per SM) all three products share one accumulator.  The tensor
// cores add each MMA's products to the accumulator with truncation, an error
// that grows with the number of MMAs and with the accumulator's magnitude:
// kept apart, the small cross terms are not truncated against the large
// high-part sum, and rounding both splits to nearest (rather than truncating
// the high part) removes their bias.
// Measured on B200 against FP64 (128 rows, 8 columns, K = 200, positive
// inputs): truncated split + one accumulator 4.5e-6, rounded split + two
// accumulators 1.1e-6 (FP32 FMA chain 2.2e-7).
//
// One 256-thread CTA per SM walks the classes round robin (classes are
// ordered largest first).  Per chunk of KC k-values: thread 0 issues one
// bulk copy per 16-byte k group (rows_c x 16 bytes) on an mbarrier; all
// threads build the B operand through the problem and split both operands into
// the no-swizzle K-major core-matrix layout (element (row, k) at
// (k / kc) LBO + (row / 8) 128 + (row % 8) 16 + (k % kc) size, kc = 16 bytes /
// element size, LBO = rows * 16, SBO = 128); thread 0 issues the MMAs (M =
// 128 rows per tile) and commits them to a second mbarrier.  Two stages
// alternate, so the next chunk's copies and operand work overlap the MMAs.
// The epilogue reads the accumulators with tcgen05.ld 32x32b (one row per
// thread, 8 columns per group) and hands each group's 8 values to the problem.
// Every wait is bounded (about a second); a wait that gives up sets status bit
// 2, lets nothing further be issued, drains what is in flight and frees the
// tensor memory.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.h"

namespace phgpu {

constexpr int kTcThreads = 256;
constexpr int kTcCtasPerSm = 3;  // 3 x 256 threads x at most 85 registers fit 64K registers
constexpr int kTcStages = 2;

// Per-launch geometry (host-computed, tc_gemm_geom).
struct TcGemmArgs {
  int MP;          // A rows padded to whole 128-row tiles (the largest class)
  int nmt;         // 128-row tiles
  int N;           // B rows (output columns): 8 per group, padded to 16
  int groups;      // column groups of 8
  int KC;          // k values per chunk (16 or 32)
  int precision;   // kSo3Tf32x3 / kSo3Bf16x3
  uint32_t a32;    // FP32 A chunk: KC * MP * 4 bytes
  uint32_t aconv;  // tf32: low parts (a32); bf16: high + low parts (a32)
  uint32_t bop;    // B operand, high + low
  uint32_t stage;
  uint32_t smem;
  uint32_t tcols;  // tensor-memory columns (high-part sums, then cross-term sums at xoff)
  uint32_t xoff;   // column offset of the cross-term accumulators
  int ctas_per_sm; // CTAs one SM runs at once (tensor and shared memory)
  unsigned long long* status;
};

// A class: rows_c rows of A (<= MP), kdim k values (a multiple of 8), its A block.
struct TcClass {
  int rows;
  int kdim;
  const float* a;
  int u0, u1;  // problem data (e.g. the orders of the class)
};

// Shared and tensor memory of a launch with KC k values per chunk; false
// when it does not fit.
inline bool tc_gemm_geom_kc(int max_rows, int groups, int precision, int KC, bool sep, TcGemmArgs* g) {
  if (precision != kSo3Tf32x3 && precision != kSo3Bf16x3) return false;
  if (groups < 1 || max_rows < 1) return false;
  g->precision = precision;
  g->groups = groups;
  g->nmt = (max_rows + 127) / 128;
  g->MP = g->nmt * 128;
  g->N = ((8 * groups + 15) / 16) * 16;
  const int nacc = sep ? 2 : 1;
  if (g->N > 256 || nacc * g->nmt * g->N > 512) return false;
  g->KC = KC;
  g->a32 = (uint32_t)KC * g->MP * 4;
  g->aconv = g->a32;
  g->bop = (uint32_t)(precision == kSo3Tf32x3 ? 8 : 4) * KC * g->N;
  g->stage = g->a32 + g->aconv + g->bop;
  g->smem = kTcStages * g->stage + 1024u;
  if (g->smem > 227u * 1024u) return false;
  g->xoff = sep ? (uint32_t)(g->nmt * g->N) : 0u;
  uint32_t c = 32;
  while (c < (uint32_t)(nacc * g->nmt * g->N)) c <<= 1;
  g->tcols = c;
  // CTAs that may share an SM: as many as the 512 tensor-memory columns hold
  // (so an allocation never waits) and the registers hold (kTcCtasPerSm, the
  // kernels' launch bound), enforced through the shared memory each CTA takes
  // (228 KB per SM, 1 KB of it reserved per CTA)
  g->ctas_per_sm = (int)(512u / c);
  if (g->ctas_per_sm > kTcCtasPerSm) g->ctas_per_sm = kTcCtasPerSm;
  const uint32_t fit = 228u * 1024u / (g->smem + 1024u);
  if ((uint32_t)g->ctas_per_sm > fit) g->ctas_per_sm = (int)(fit > 0 ? fit : 1);
  const uint32_t floor_smem = 228u * 1024u / (uint32_t)(g->ctas_per_sm + 1) + 1u;
  if (g->smem < floor_smem) g->smem = floor_smem;
  return true;
}

// The launch geometry: chunk = 16 or 32 k values, or 0 for the one of the two
// that lets more CTAs share an SM (32 on a tie).  sep: the cross terms
// accumulate in tensor-memory columns of their own (see the file comment).
inline bool tc_gemm_geom(int max_rows, int groups, int precision, int chunk, bool sep, TcGemmArgs* g) {
  if (chunk) return tc_gemm_geom_kc(max_rows, groups, precision, chunk, sep, g);
  TcGemmArgs a, b;
  const bool ok32 = tc_gemm_geom_kc(max_rows, groups, precision, 32, sep, &a);
  const bool ok16 = tc_gemm_geom_kc(max_rows, groups, precision, 16, sep, &b);
  if (!ok32 && !ok16) return false;
  *g = ok32 && (!ok16 || a.ctas_per_sm >= b.ctas_per_sm) ? a : b;
  return true;
}

#ifdef __CUDACC__

__device__ __forceinline__ uint32_t tc_smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

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
// another thread gave up and honour_abort) and returns false.
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

// FP32 bits rounded to the nearest TF32 value (10 stored mantissa bits; ties
// away from zero), the form kind::tf32 reads.
__device__ __forceinline__ uint32_t tf32_rn(uint32_t x) { return (x + 0x1000u) & 0xFFFFE000u; }

__device__ __forceinline__ float tf32_lo(float x, uint32_t hi) {
  return __uint_as_float(tf32_rn(__float_as_uint(x - __uint_as_float(hi))));
}

// The GEMMs of every class of `prob` (see the file comment).  P provides
//   int classes() const;
//   TcClass cls(int c) const;
//   void bvals(const TcClass& c, int group, int k, float v[8]) const;   // zero for k >= the real length
//   void store(const TcClass& c, int group, int row, const float v[8]) const;
template <int PREC, class P>
__device__ __forceinline__ void tc_class_gemm(const TcGemmArgs& g, const P& prob) {
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
  const int MP = g.MP, N = g.N, KC = g.KC;
  const uint32_t lboA = (uint32_t)MP * 16, lboB = (uint32_t)N * 16;

  // zero every operand buffer once: padding rows and columns stay zero
  for (uint32_t e = tid; e < kTcStages * g.stage / 16; e += kTcThreads)
    reinterpret_cast<uint4*>(smem)[e] = make_uint4(0u, 0u, 0u, 0u);
  if (tid == 0) {
    for (int b = 0; b < 4; ++b) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem_addr(&bars[b])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    *s_abort = 0;
    for (int b = 0; b < 4; ++b) s_pending[b] = 0;
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem_addr(s_tmem)),
                 "r"(g.tcols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;
  const uint32_t idesc = umma_idesc(PREC == kSo3Tf32x3 ? 2u : 1u, (uint32_t)N);
  const int ncls = prob.classes();

  uint32_t it = 0;  // chunks processed by this CTA (stage = it & 1)
  for (int c = blockIdx.x; c < ncls; c += gridDim.x) {
    const TcClass cl = prob.cls(c);
    const int rows = cl.rows;
    const int nch = (cl.kdim + KC - 1) / KC;
    for (int ch = 0; ch < nch; ++ch, ++it) {
      const int s = it & 1;
      uint8_t* stage = smem + s * g.stage;
      float* A32 = reinterpret_cast<float*>(stage);
      uint8_t* AX = stage + g.a32;
      uint8_t* BH = stage + g.a32 + g.aconv;
      uint8_t* BL = BH + g.bop / 2;
      const int kcc = min(KC, cl.kdim - ch * KC) / 4;    // 16-byte k groups of this chunk
      const int ksteps = (kcc * 4 + KSTEP - 1) / KSTEP;  // MMAs along k
      const int kread = ksteps * KSTEP;                  // k values the MMAs read
      // stage s was last read by the MMAs of chunk it - 2
      if (it >= 2) tc_wait(tc_smem_addr(&bars[2 + s]), ((it >> 1) - 1) & 1, s_abort, true);
      if (tid == 0) s_pending[2 + s] = 0;
      if (tid == 0 && !*s_abort) {
        const uint32_t bytes = (uint32_t)kcc * rows * 16;
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc_smem_addr(&bars[s])),
                     "r"(bytes)
                     : "memory");
        for (int cc = 0; cc < kcc; ++cc) {
          const float* src = cl.a + ((size_t)(ch * KC / 4 + cc) * rows) * 4;
          asm volatile(
              "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                  tc_smem_addr(A32 + (size_t)cc * MP * 4)),
              "l"(src), "r"((uint32_t)rows * 16), "r"(tc_smem_addr(&bars[s]))
              : "memory");
        }
        s_pending[s] = 1 + (int)((it >> 1) & 1);
      }
      // B operand: rows j = 8 group + u, the chunk's k values
      const int k0 = ch * KC;
      for (int e = tid; e < g.groups * kread; e += kTcThreads) {
        const int grp = e / kread, il = e - grp * kread;
        float vals[8];
        prob.bvals(cl, grp, k0 + il, vals);
        const uint32_t off = (uint32_t)(il / KCE) * lboB + (uint32_t)(il % KCE) * ESZ;
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const uint32_t o = off + (uint32_t)(8 * grp + u) * 16;
          if constexpr (PREC == kSo3Tf32x3) {
            const uint32_t hi = tf32_rn(__float_as_uint(vals[u]));
            *reinterpret_cast<uint32_t*>(BH + o) = hi;
            *reinterpret_cast<float*>(BL + o) = tf32_lo(vals[u], hi);
          } else {
            const __nv_bfloat16 hi = __float2bfloat16_rn(vals[u]);
            *reinterpret_cast<__nv_bfloat16*>(BH + o) = hi;
            *reinterpret_cast<__nv_bfloat16*>(BL + o) = __float2bfloat16_rn(vals[u] - __bfloat162float(hi));
          }
        }
      }
      tc_wait(tc_smem_addr(&bars[s]), (it >> 1) & 1, s_abort, true);
      if (tid == 0) s_pending[s] = 0;
      // split the A chunk (rows < rows; the others keep zeros or an earlier
      // class's values, which only reach accumulator rows that are not stored)
      if constexpr (PREC == kSo3Tf32x3) {
        uint4* hi = reinterpret_cast<uint4*>(A32);
        float4* lo = reinterpret_cast<float4*>(AX);
        // (k group, row) walked without a per-element division
        for (int cc = 0; cc < kcc; ++cc) {
          for (int row = tid; row < rows; row += kTcThreads) {
            const size_t idx = (size_t)cc * MP + row;
            const uint4 x = hi[idx];
            const uint4 h = make_uint4(tf32_rn(x.x), tf32_rn(x.y), tf32_rn(x.z), tf32_rn(x.w));
            hi[idx] = h;
            lo[idx] = make_float4(tf32_lo(__uint_as_float(x.x), h.x), tf32_lo(__uint_as_float(x.y), h.y),
                                  tf32_lo(__uint_as_float(x.z), h.z), tf32_lo(__uint_as_float(x.w), h.w));
          }
        }
      } else {
        uint4* hi16 = reinterpret_cast<uint4*>(AX);
        uint4* lo16 = reinterpret_cast<uint4*>(AX + g.aconv / 2);
        const float4* src = reinterpret_cast<const float4*>(A32);
        for (int c16 = 0; c16 < kread / 8; ++c16) {
          for (int row = tid; row < rows; row += kTcThreads) {
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
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      if (tid == 0 && !*s_abort) {
        tc_fence_after();
        const uint32_t aH = PREC == kSo3Tf32x3 ? tc_smem_addr(A32) : tc_smem_addr(AX);
        const uint32_t aL = PREC == kSo3Tf32x3 ? tc_smem_addr(AX) : tc_smem_addr(AX + g.aconv / 2);
        const uint32_t bH = tc_smem_addr(BH), bL = tc_smem_addr(BL);
        const int ntile = (rows + 127) / 128;
        for (int ks = 0; ks < ksteps; ++ks) {
          for (int t = 0; t < ntile; ++t) {
            const uint32_t dt = tmem + (uint32_t)(t * N);
            const uint32_t ao = (uint32_t)ks * 2u * lboA + (uint32_t)t * 2048u;
            const uint32_t bo = (uint32_t)ks * 2u * lboB;
            const uint32_t first = (ch == 0 && ks == 0) ? 0u : 1u;
            umma<PREC>(dt, umma_desc(aH + ao, lboA, 128), umma_desc(bH + bo, lboB, 128), idesc, first);
            umma<PREC>(dt + g.xoff, umma_desc(aH + ao, lboA, 128), umma_desc(bL + bo, lboB, 128), idesc,
                       g.xoff ? first : 1u);
            umma<PREC>(dt + g.xoff, umma_desc(aL + ao, lboA, 128), umma_desc(bH + bo, lboB, 128), idesc, 1u);
          }
        }
        umma_commit(tc_smem_addr(&bars[2 + s]));
        s_pending[2 + s] = 1 + (int)((it >> 1) & 1);
      }
    }
    // epilogue: the last chunk's MMAs complete every accumulation of the class
    const uint32_t last = it - 1;
    tc_wait(tc_smem_addr(&bars[2 + (last & 1)]), (last >> 1) & 1, s_abort, true);
    tc_fence_after();
    const int qd = warp & 3;
    const int ntile = (rows + 127) / 128;
    for (int t = warp >> 2; t < ntile; t += 2) {
      const int row = t * 128 + qd * 32 + lane;
      for (int grp = 0; grp < g.groups; ++grp) {
        uint32_t v[8], w[8] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
        const uint32_t ta = tmem + ((uint32_t)(qd * 32) << 16) + (uint32_t)(t * N + 8 * grp);
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                     : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                     : "r"(ta));
        if (g.xoff)  // block-uniform
          asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                       : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]), "=r"(w[4]), "=r"(w[5]), "=r"(w[6]), "=r"(w[7])
                       : "r"(ta + g.xoff));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (row < rows && !*s_abort) {
          float f[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) f[u] = __uint_as_float(v[u]) + __uint_as_float(w[u]);
          prob.store(cl, grp, row, f);
        }
      }
    }
    tc_fence_before();
    __syncthreads();
  }
  // leave nothing in flight, then release the tensor memory
  if (tid == 0) {
    for (int b = 0; b < 4; ++b)
      if (s_pending[b]) tc_wait(tc_smem_addr(&bars[b]), (uint32_t)(s_pending[b] - 1), s_abort, false);
    if (*s_abort) atomicOr(g.status, 2ull);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(g.tcols) : "memory");
}

#endif  // __CUDACC__

}  // namespace phgpu
