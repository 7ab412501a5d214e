// Register-tail FFT engine for the fixed lengths of the workloads (FP32).
//
// A length N is split as N = R0 (* R1) * M: one or two in-place radix stages
// through shared memory, then every block of M contiguous positions is
// transformed by one thread in registers, where all twiddles are compile-time
// constants.  The factorisation and the resulting digit-reversed order are the
// same as the host planner's and fft.cuh's (radix 8 first, then 4, 2, 5, 3),
// so positions and frequencies agree with fixed_freq2pos / fixed_pos2freq.
//
// Thread mapping: the block has T threads (T a multiple of every stage's
// butterfly count).  In each shared-memory stage a thread keeps one butterfly
// position -- hence one set of twiddles, loaded once -- and walks over the
// transforms; neighbouring threads take neighbouring transforms (columns) or
// neighbouring butterflies (rows), which keeps shared-memory accesses
// conflict-free.
#pragma once

#include "fft.cuh"

namespace phgpu {

// ---------------------------------------------------------------- constexpr twiddles

constexpr double kPiD = 3.14159265358979323846264338327950288;

constexpr double cx_sin_taylor(double x) {
  double term = x, sum = x;
  for (int n = 1; n < 30; ++n) {
    term *= -x * x / ((2.0 * n) * (2.0 * n + 1.0));
    sum += term;
  }
  return sum;
}
constexpr double cx_reduce(double a) {
  while (a > kPiD) a -= 2.0 * kPiD;
  while (a < -kPiD) a += 2.0 * kPiD;
  return a;
}
constexpr double cx_sin(double a) { return cx_sin_taylor(cx_reduce(a)); }
constexpr double cx_cos(double a) { return cx_sin_taylor(cx_reduce(a + 0.5 * kPiD)); }

// w_M^e = exp(-2 pi i e / M) for e in [0, M)
template <int M>
struct ConstTw {
  float re[M], im[M];
  constexpr ConstTw() : re(), im() {
    for (int e = 0; e < M; ++e) {
      re[e] = (float)cx_cos(-2.0 * kPiD * e / M);
      im[e] = (float)cx_sin(-2.0 * kPiD * e / M);
    }
  }
};

template <int M>
__device__ __forceinline__ float2 ctw(int e) {
  constexpr ConstTw<M> t;
  return make_float2(t.re[e], t.im[e]);
}

// ---------------------------------------------------------------- register blocks

// In-register DIF transform of M points (M = RA * RB or a single radix);
// output in the digit-reversed order of the (RA, RB) factorisation.
template <int RA, int RB, bool INV, bool PK = true>
__device__ __forceinline__ void reg_block(float2 (&x)[RA * RB]) {
  constexpr int M = RA * RB;
  if constexpr (RB == 1) {
    dft_small<RA, INV, PK>(x);
  } else if constexpr (!INV) {
    // radix RA over stride RB, twiddle w_M^{j2 k1}
#pragma unroll
    for (int j2 = 0; j2 < RB; ++j2) {
      float2 v[RA];
#pragma unroll
      for (int j1 = 0; j1 < RA; ++j1) v[j1] = x[j2 + RB * j1];
      dft_small<RA, false, PK>(v);
#pragma unroll
      for (int k1 = 0; k1 < RA; ++k1) x[j2 + RB * k1] = (j2 * k1 == 0) ? v[k1] : cmul(v[k1], ctw<M>((j2 * k1) % M));
    }
    // RA blocks of RB contiguous points
#pragma unroll
    for (int k1 = 0; k1 < RA; ++k1) {
      float2 v[RB];
#pragma unroll
      for (int j = 0; j < RB; ++j) v[j] = x[RB * k1 + j];
      dft_small<RB, false, PK>(v);
#pragma unroll
      for (int j = 0; j < RB; ++j) x[RB * k1 + j] = v[j];
    }
  } else {
#pragma unroll
    for (int k1 = 0; k1 < RA; ++k1) {
      float2 v[RB];
#pragma unroll
      for (int j = 0; j < RB; ++j) v[j] = x[RB * k1 + j];
      dft_small<RB, true, PK>(v);
#pragma unroll
      for (int j = 0; j < RB; ++j) x[RB * k1 + j] = v[j];
    }
#pragma unroll
    for (int j2 = 0; j2 < RB; ++j2) {
      float2 v[RA];
#pragma unroll
      for (int j1 = 0; j1 < RA; ++j1) {
        const float2 a = x[j2 + RB * j1];
        v[j1] = (j2 * j1 == 0) ? a : cmul(a, cconj(ctw<M>((j2 * j1) % M)));
      }
      dft_small<RA, true, PK>(v);
#pragma unroll
      for (int k1 = 0; k1 < RA; ++k1) x[j2 + RB * k1] = v[k1];
    }
  }
}

// ---------------------------------------------------------------- plans

// N = S0 (* S1) * (TA * TB): shared-memory radices S0, S1 (S1 = 1: none), then
// a register block of TA * TB points.
template <int N>
struct Tail {
  static constexpr bool ok = false;
};
template <> struct Tail<32>  { static constexpr bool ok = true; static constexpr int S0 = 8, S1 = 1, TA = 4, TB = 1; };
template <> struct Tail<64>  { static constexpr bool ok = true; static constexpr int S0 = 8, S1 = 1, TA = 8, TB = 1; };
template <> struct Tail<100> { static constexpr bool ok = true; static constexpr int S0 = 4, S1 = 1, TA = 5, TB = 5; };
template <> struct Tail<128> { static constexpr bool ok = true; static constexpr int S0 = 8, S1 = 1, TA = 8, TB = 2; };
template <> struct Tail<200> { static constexpr bool ok = true; static constexpr int S0 = 8, S1 = 1, TA = 5, TB = 5; };
template <> struct Tail<256> { static constexpr bool ok = true; static constexpr int S0 = 8, S1 = 1, TA = 8, TB = 4; };
template <> struct Tail<512> { static constexpr bool ok = true; static constexpr int S0 = 8, S1 = 8, TA = 8, TB = 1; };

// Threads per block that divides every stage's butterfly count.
template <int N>
constexpr int tail_threads() {
  return (N == 200 || N == 100) ? 1000 : 1024;
}

// One shared-memory stage (radix R, block length L) with a per-thread fixed
// butterfly position.  COL: transforms are columns (element stride `stride`,
// transform t at offset t), neighbouring threads take neighbouring columns;
// rows: transform t at t * stride, neighbouring threads take neighbouring
// butterflies of the same row.
template <int N, int R, int L, bool INV, bool COL, bool PK = true>
__device__ __forceinline__ void tail_smem_stage(float2* buf, int ntrans, int stride, const float2* __restrict__ tw,
                                                int tid, int T, const int* rowmap = nullptr) {
  constexpr int m = L / R;
  constexpr int nb = N / R;  // butterflies per transform
  constexpr int twstep = N / L;
  const int lanes = T / nb;  // threads sharing one butterfly position
  int b, t0;
  if (COL) {
    b = tid / lanes;
    t0 = tid - b * lanes;
  } else {
    b = tid % nb;
    t0 = tid / nb;
  }
  if (b >= nb || t0 >= lanes) return;
  const int blk = b / m, j2 = b - (b / m) * m;
  float2 w[R];
#pragma unroll
  for (int k = 1; k < R; ++k) {
    w[k] = __ldg(&tw[twstep * j2 * k]);
    if (INV) w[k] = cconj(w[k]);
  }
  const int off = blk * L + j2;
  const int es = COL ? m * stride : m;
  for (int t = t0; t < ntrans; t += lanes) {
    const int tt = (!COL && rowmap) ? rowmap[t] : t;
    float2* base = COL ? buf + tt + (size_t)off * stride : buf + (size_t)tt * stride + off;
    float2 x[R];
#pragma unroll
    for (int j = 0; j < R; ++j) x[j] = base[j * es];
    if (INV) {
#pragma unroll
      for (int k = 1; k < R; ++k) x[k] = cmul(x[k], w[k]);
      dft_small<R, true, PK>(x);
    } else {
      dft_small<R, false, PK>(x);
#pragma unroll
      for (int k = 1; k < R; ++k) x[k] = cmul(x[k], w[k]);
    }
#pragma unroll
    for (int j = 0; j < R; ++j) base[j * es] = x[j];
  }
}

// Register blocks: neighbouring threads take neighbouring transforms (rows
// need an odd-ish row stride, e.g. N + 1, to stay conflict-free).
template <int N, bool INV, bool COL, bool PK = true>
__device__ __forceinline__ void tail_reg_stage(float2* buf, int ntrans, int stride, int tid, int T,
                                               const int* rowmap = nullptr) {
  using P = Tail<N>;
  constexpr int M = P::TA * P::TB;
  constexpr int nbk = N / M;  // register blocks per transform
  const int lanes = T / nbk;
  const int bk = tid / lanes;
  if (bk >= nbk) return;
  for (int t = tid - bk * lanes; t < ntrans; t += lanes) {
    const int tt = (!COL && rowmap) ? rowmap[t] : t;
    float2* base = COL ? buf + tt + (size_t)(bk * M) * stride : buf + (size_t)tt * stride + bk * M;
    const int es = COL ? stride : 1;
    float2 x[M];
#pragma unroll
    for (int j = 0; j < M; ++j) x[j] = base[j * es];
    reg_block<P::TA, P::TB, INV, PK>(x);
#pragma unroll
    for (int j = 0; j < M; ++j) base[j * es] = x[j];
  }
}

// Batched in-place transform.  Same position convention as fft_fixed<N>.
// Caller synchronises before; ends with __syncthreads().  T = blockDim.x must
// be a multiple of every stage's butterfly count (tail_threads<N>() is).
// Rows only: with rowmap, transform t is row rowmap[t] (t < ntrans), which
// lets a caller transform just the rows that are not all zero.
// NT > 0: the block has exactly NT threads (the per-thread split folds to
// constants); NT = 0: blockDim.x.
template <int N, bool INV, bool COL, bool PK = true, int NT = 0>
__device__ __forceinline__ void fft_tail(float2* buf, int ntrans, int stride, const float2* __restrict__ tw,
                                         const int* rowmap = nullptr) {
  using P = Tail<N>;
  static_assert(P::ok, "no register-tail plan for this length");
  const int tid = threadIdx.x, T = NT > 0 ? NT : (int)blockDim.x;
  if constexpr (!INV) {
    tail_smem_stage<N, P::S0, N, false, COL, PK>(buf, ntrans, stride, tw, tid, T, rowmap);
    __syncthreads();
    if constexpr (P::S1 > 1) {
      tail_smem_stage<N, P::S1, N / P::S0, false, COL, PK>(buf, ntrans, stride, tw, tid, T, rowmap);
      __syncthreads();
    }
    tail_reg_stage<N, false, COL, PK>(buf, ntrans, stride, tid, T, rowmap);
    __syncthreads();
  } else {
    tail_reg_stage<N, true, COL, PK>(buf, ntrans, stride, tid, T, rowmap);
    __syncthreads();
    if constexpr (P::S1 > 1) {
      tail_smem_stage<N, P::S1, N / P::S0, true, COL, PK>(buf, ntrans, stride, tw, tid, T, rowmap);
      __syncthreads();
    }
    tail_smem_stage<N, P::S0, N, true, COL, PK>(buf, ntrans, stride, tw, tid, T, rowmap);
    __syncthreads();
  }
}

}  // namespace phgpu
