// In-place mixed-radix FFT on shared-memory batches (FP32, sm_100a).
//
// Forward transforms run decimation-in-frequency and leave the spectrum in
// mixed-radix digit-reversed order; inverse transforms run decimation-in-time
// from that order back to natural order.  A forward/inverse pair therefore
// needs no permutation pass, and the pointwise work between them (channel
// fusion, cross power) only maps positions to frequencies with fft_pos2freq.
//
// Stage s has radix r_s and block length L_s = n / (r_0 ... r_{s-1}); a
// butterfly reads r_s elements spaced m_s = L_s / r_s apart and applies the
// twiddle w_n^{(n / L_s) j2 k1}.  Twiddles come from a table w[t] =
// exp(-2 pi i t / n) computed in double precision on the host.
#pragma once

#include "common.cuh"

namespace phgpu {

constexpr int kMaxFftStages = 16;

struct FftPlan {
  int n;
  int nstage;
  int radix[kMaxFftStages];
  int L[kMaxFftStages];
  const float2* tw;  // n entries
};

// Position after a forward (DIF) transform of frequency k.
__host__ __device__ inline int fft_freq2pos(int k, const FftPlan& p) {
  int pos = 0, L = p.n;
  for (int s = 0; s < p.nstage; ++s) {
    const int r = p.radix[s];
    const int m = L / r;
    pos += (k % r) * m;
    k /= r;
    L = m;
  }
  return pos;
}

// Frequency stored at position pos after a forward (DIF) transform.
__host__ __device__ inline int fft_pos2freq(int pos, const FftPlan& p) {
  int k = 0, mult = 1, L = p.n;
  for (int s = 0; s < p.nstage; ++s) {
    const int r = p.radix[s];
    const int m = L / r;
    k += (pos / m) * mult;
    pos %= m;
    mult *= r;
    L = m;
  }
  return k;
}

template <int R, bool INV>
__device__ __forceinline__ void dft_small(float2 (&x)[R]) {
  constexpr float sg = INV ? 1.0f : -1.0f;  // exponent sign
  if constexpr (R == 2) {
    const float2 a = x[0], b = x[1];
    x[0] = cadd(a, b);
    x[1] = csub(a, b);
  } else if constexpr (R == 3) {
    const float s3 = 0.86602540378443864676f;
    const float2 t1 = cadd(x[1], x[2]);
    const float2 t2 = csub(x[1], x[2]);
    const float2 y0 = cadd(x[0], t1);
    const float2 m1 = make_float2(x[0].x - 0.5f * t1.x, x[0].y - 0.5f * t1.y);
    // i * sg * s3 * t2
    const float2 m2 = make_float2(-sg * s3 * t2.y, sg * s3 * t2.x);
    x[0] = y0;
    x[1] = cadd(m1, m2);
    x[2] = csub(m1, m2);
  } else if constexpr (R == 4) {
    const float2 t0 = cadd(x[0], x[2]);
    const float2 t1 = csub(x[0], x[2]);
    const float2 t2 = cadd(x[1], x[3]);
    const float2 d = csub(x[1], x[3]);
    const float2 t3 = make_float2(-sg * d.y, sg * d.x);  // i*sg*d
    x[0] = cadd(t0, t2);
    x[2] = csub(t0, t2);
    x[1] = cadd(t1, t3);
    x[3] = csub(t1, t3);
  } else if constexpr (R == 5) {
    const float c1 = 0.30901699437494742410f, c2 = -0.80901699437494742410f;
    const float s1 = 0.95105651629515357212f, s2 = 0.58778525229247312917f;
    const float2 t1 = cadd(x[1], x[4]), t2 = cadd(x[2], x[3]);
    const float2 t3 = csub(x[1], x[4]), t4 = csub(x[2], x[3]);
    const float2 y0 = cadd(x[0], cadd(t1, t2));
    const float2 a1 = make_float2(x[0].x + c1 * t1.x + c2 * t2.x, x[0].y + c1 * t1.y + c2 * t2.y);
    const float2 a2 = make_float2(x[0].x + c2 * t1.x + c1 * t2.x, x[0].y + c2 * t1.y + c1 * t2.y);
    const float2 b1 = make_float2(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y);
    const float2 b2 = make_float2(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y);
    // y1 = a1 + i*sg*b1, y4 = a1 - i*sg*b1, y2 = a2 + i*sg*b2, y3 = a2 - i*sg*b2
    const float2 ib1 = make_float2(-sg * b1.y, sg * b1.x);
    const float2 ib2 = make_float2(-sg * b2.y, sg * b2.x);
    x[0] = y0;
    x[1] = cadd(a1, ib1);
    x[4] = csub(a1, ib1);
    x[2] = cadd(a2, ib2);
    x[3] = csub(a2, ib2);
  } else if constexpr (R == 8) {
    float2 e[4] = {x[0], x[2], x[4], x[6]};
    float2 o[4] = {x[1], x[3], x[5], x[7]};
    dft_small<4, INV>(e);
    dft_small<4, INV>(o);
    const float h = 0.70710678118654752440f;
    // w8^k = exp(sg * i * pi k / 4)
    const float2 w1 = make_float2(h, sg * h);
    const float2 w3 = make_float2(-h, sg * h);
    const float2 o1 = cmul(o[1], w1);
    const float2 o2 = make_float2(-sg * o[2].y, sg * o[2].x);
    const float2 o3 = cmul(o[3], w3);
    x[0] = cadd(e[0], o[0]);
    x[4] = csub(e[0], o[0]);
    x[1] = cadd(e[1], o1);
    x[5] = csub(e[1], o1);
    x[2] = cadd(e[2], o2);
    x[6] = csub(e[2], o2);
    x[3] = cadd(e[3], o3);
    x[7] = csub(e[3], o3);
  } else {
    // generic small odd prime
    float2 y[R];
#pragma unroll
    for (int k = 0; k < R; ++k) {
      float2 acc = x[0];
#pragma unroll
      for (int j = 1; j < R; ++j) {
        float s, c;
        sincospif(2.0f * (float)((j * k) % R) / (float)R, &s, &c);
        const float2 w = make_float2(c, sg * s);
        acc = cadd(acc, cmul(x[j], w));
      }
      y[k] = acc;
    }
#pragma unroll
    for (int k = 0; k < R; ++k) x[k] = y[k];
  }
}

// One radix-R stage over `ntrans` transforms; element i of transform t is at
// buf[t * tstride + i * estride].  Threads iterate butterflies with the
// transform index fastest when estride != 1 (columns), so neighbouring
// threads touch neighbouring shared-memory words.
template <int R, bool INV>
__device__ __forceinline__ void fft_stage(float2* buf, int ntrans, int tstride, int estride, int n,
                                          int L, const float2* __restrict__ tw, int tid,
                                          int nthr) {
  const int m = L / R;
  const int nb = n / R;
  const int total = ntrans * nb;
  const int twstep = n / L;
  const int es = m * estride;
  for (int it = tid; it < total; it += nthr) {
    int t, bf;
    if (estride == 1) {
      t = it / nb;
      bf = it - t * nb;
    } else {
      bf = it / ntrans;
      t = it - bf * ntrans;
    }
    const int blk = bf / m;
    const int j2 = bf - blk * m;
    float2* base = buf + t * tstride + (blk * L + j2) * estride;
    float2 x[R];
#pragma unroll
    for (int j = 0; j < R; ++j) x[j] = base[j * es];
    if (INV) {
#pragma unroll
      for (int k = 1; k < R; ++k) x[k] = cmul(x[k], cconj(__ldg(&tw[twstep * j2 * k])));
      dft_small<R, true>(x);
    } else {
      dft_small<R, false>(x);
#pragma unroll
      for (int k = 1; k < R; ++k) x[k] = cmul(x[k], __ldg(&tw[twstep * j2 * k]));
    }
#pragma unroll
    for (int j = 0; j < R; ++j) base[j * es] = x[j];
  }
}

// Radix-R stage for any R <= kMaxGenericRadix (rare lengths with a large prime
// factor, e.g. 201 = 3 * 67): the O(R^2) butterfly spread over threads.  A
// work item is kGenericOuts outputs of kGenericBfs butterflies, summed from
// the inputs in shared memory with table twiddles (index j * k mod R kept
// incrementally).
// Butterflies are processed in rounds of whole butterflies: every item of a
// round reads, the block synchronises, then writes, so the in-place update
// never overwrites an input another item still needs.  The inverse stage
// first multiplies its inputs by the conjugate twiddles in place.  Contains
// __syncthreads(): every thread of the block must call it.
constexpr int kMaxGenericRadix = 128;
constexpr int kGenericOuts = 4;
constexpr int kGenericBfs = 4;

__device__ __forceinline__ float2* generic_base(float2* buf, int bfi, int ntrans, int nb, int m, int L, int tstride,
                                                int estride, int& j2) {
  int t, bf;
  if (estride == 1) {
    t = bfi / nb;
    bf = bfi - t * nb;
  } else {
    bf = bfi / ntrans;
    t = bfi - bf * ntrans;
  }
  const int blk = bf / m;
  j2 = bf - blk * m;
  return buf + t * tstride + (blk * L + j2) * estride;
}

template <bool INV>
__device__ __noinline__ void fft_stage_generic(float2* buf, int R, int ntrans, int tstride, int estride, int n,
                                               int L, const float2* __restrict__ tw, int tid, int nthr) {
  const int m = L / R;
  const int nb = n / R;
  const int nbf = ntrans * nb;  // butterflies
  const int twstep = n / L;
  const int es = m * estride;
  const int rstep = n / R;
  const int ng = (R + kGenericOuts - 1) / kGenericOuts;  // output groups per butterfly
  if (INV) {
    for (int it = tid; it < nbf * R; it += nthr) {
      const int bfi = it / R, j = it - bfi * R;
      if (j == 0) continue;
      int j2;
      float2* base = generic_base(buf, bfi, ntrans, nb, m, L, tstride, estride, j2);
      base[j * es] = cmul(base[j * es], cconj(__ldg(&tw[twstep * j2 * j])));
    }
    __syncthreads();
  }
  // an item: kGenericOuts outputs of kGenericBfs consecutive butterflies (a
  // twiddle load serves every butterfly, an input load every output)
  const int nbg = (nbf + kGenericBfs - 1) / kGenericBfs;  // butterfly groups
  const int grp_round = max(1, nthr / ng);
  for (int g0 = 0; g0 < nbg; g0 += grp_round) {
    const int nitems = min(grp_round, nbg - g0) * ng;
    const bool active = tid < nitems;
    float2 acc[kGenericBfs][kGenericOuts];
    float2* base[kGenericBfs];
    int j2[kGenericBfs];
    bool live[kGenericBfs];
    int k0 = 0;
    if (active) {
      const int grp = g0 + tid / ng;
      k0 = (tid - (tid / ng) * ng) * kGenericOuts;
#pragma unroll
      for (int u = 0; u < kGenericBfs; ++u) {
        const int bfi = grp * kGenericBfs + u;
        live[u] = bfi < nbf;
        base[u] = generic_base(buf, live[u] ? bfi : 0, ntrans, nb, m, L, tstride, estride, j2[u]);
        const float2 x0 = base[u][0];
#pragma unroll
        for (int i = 0; i < kGenericOuts; ++i) acc[u][i] = x0;
      }
      int kk[kGenericOuts], mi[kGenericOuts];
#pragma unroll
      for (int i = 0; i < kGenericOuts; ++i) {
        kk[i] = k0 + i < R ? k0 + i : 0;  // padding outputs of the last group stay at index 0
        mi[i] = 0;
      }
      for (int j = 1; j < R; ++j) {
        float2 xj[kGenericBfs];
#pragma unroll
        for (int u = 0; u < kGenericBfs; ++u) xj[u] = base[u][j * es];
#pragma unroll
        for (int i = 0; i < kGenericOuts; ++i) {
          mi[i] += kk[i];
          if (mi[i] >= R) mi[i] -= R;
          float2 w = __ldg(&tw[rstep * mi[i]]);
          if (INV) w = cconj(w);
#pragma unroll
          for (int u = 0; u < kGenericBfs; ++u) acc[u][i] = cadd(acc[u][i], cmul(xj[u], w));
        }
      }
    }
    __syncthreads();
    if (active) {
#pragma unroll
      for (int u = 0; u < kGenericBfs; ++u) {
        if (!live[u]) continue;
#pragma unroll
        for (int i = 0; i < kGenericOuts; ++i) {
          const int k = k0 + i;
          if (k < R) {
            float2 a = acc[u][i];
            if (!INV && k > 0) a = cmul(a, __ldg(&tw[twstep * j2[u] * k]));
            base[u][k * es] = a;
          }
        }
      }
    }
    __syncthreads();
  }
}

// Batched in-place transform.  Caller synchronises before; the function ends
// with __syncthreads().  All threads of the block must call it.
template <bool INV>
__device__ void fft_smem(float2* buf, int ntrans, int tstride, int estride, const FftPlan& p) {
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nthr = blockDim.x * blockDim.y * blockDim.z;
  for (int si = 0; si < p.nstage; ++si) {
    const int s = INV ? (p.nstage - 1 - si) : si;
    const int L = p.L[s];
    switch (p.radix[s]) {
      case 2: fft_stage<2, INV>(buf, ntrans, tstride, estride, p.n, L, p.tw, tid, nthr); break;
      case 3: fft_stage<3, INV>(buf, ntrans, tstride, estride, p.n, L, p.tw, tid, nthr); break;
      case 4: fft_stage<4, INV>(buf, ntrans, tstride, estride, p.n, L, p.tw, tid, nthr); break;
      case 5: fft_stage<5, INV>(buf, ntrans, tstride, estride, p.n, L, p.tw, tid, nthr); break;
      case 7: fft_stage<7, INV>(buf, ntrans, tstride, estride, p.n, L, p.tw, tid, nthr); break;
      case 8: fft_stage<8, INV>(buf, ntrans, tstride, estride, p.n, L, p.tw, tid, nthr); break;
      case 11: fft_stage<11, INV>(buf, ntrans, tstride, estride, p.n, L, p.tw, tid, nthr); break;
      case 13: fft_stage<13, INV>(buf, ntrans, tstride, estride, p.n, L, p.tw, tid, nthr); break;
      default:
        fft_stage_generic<INV>(buf, p.radix[s], ntrans, tstride, estride, p.n, L, p.tw, tid, nthr);
        break;
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------------
// Compile-time plans for the lengths the workloads use.  The factorisation
// matches the host planner (radix 8 first, then 4, 2, 5, 3) so positions and
// frequencies agree with the runtime plan of the same length.
template <int N>
struct FixedFft {
  static constexpr int count = 0;
};
template <>
struct FixedFft<16> {
  static constexpr int count = 2;
  static constexpr int r[2] = {8, 2};
};
template <>
struct FixedFft<32> {
  static constexpr int count = 2;
  static constexpr int r[2] = {8, 4};
};
template <>
struct FixedFft<100> {
  static constexpr int count = 3;
  static constexpr int r[3] = {4, 5, 5};
};
template <>
struct FixedFft<64> {
  static constexpr int count = 2;
  static constexpr int r[2] = {8, 8};
};
template <>
struct FixedFft<128> {
  static constexpr int count = 3;
  static constexpr int r[3] = {8, 8, 2};
};
template <>
struct FixedFft<200> {
  static constexpr int count = 3;
  static constexpr int r[3] = {8, 5, 5};
};
template <>
struct FixedFft<256> {
  static constexpr int count = 3;
  static constexpr int r[3] = {8, 8, 4};
};
template <>
struct FixedFft<512> {
  static constexpr int count = 3;
  static constexpr int r[3] = {8, 8, 8};
};
template <>
struct FixedFft<320> {  // 2 bw_out for bw_out = 160 (B = 150 with zero padding 10)
  static constexpr int count = 3;
  static constexpr int r[3] = {8, 8, 5};
};

template <int N>
constexpr bool fixed_fft_supported() {
  return FixedFft<N>::count > 0;
}

template <int N, int S>
__host__ __device__ constexpr int fixed_L() {
  if constexpr (S == 0) {
    return N;
  } else {
    return fixed_L<N, S - 1>() / FixedFft<N>::r[S - 1];
  }
}

template <int N, int S = 0>
__host__ __device__ __forceinline__ int fixed_freq2pos(int k) {
  if constexpr (S >= FixedFft<N>::count) {
    return 0;
  } else {
    constexpr int r = FixedFft<N>::r[S];
    constexpr int m = fixed_L<N, S>() / r;
    return (k % r) * m + fixed_freq2pos<N, S + 1>(k / r);
  }
}

template <int N, int S = 0>
__host__ __device__ __forceinline__ int fixed_pos2freq(int pos) {
  if constexpr (S >= FixedFft<N>::count) {
    return 0;
  } else {
    constexpr int r = FixedFft<N>::r[S];
    constexpr int m = fixed_L<N, S>() / r;
    return (pos / m) + r * fixed_pos2freq<N, S + 1>(pos % m);
  }
}

// One stage with compile-time length, radix and block length.  LOG2T >= 0:
// column mode with 2^LOG2T transforms and the transform index fastest;
// LOG2T < 0: row mode (estride 1), butterfly index fastest.
template <int N, int R, int L, bool INV, int LOG2T>
__device__ __forceinline__ void fixed_stage(float2* buf, int ntrans, int tstride, int estride,
                                            const float2* __restrict__ tw, int tid, int nthr) {
  constexpr int m = L / R;
  constexpr int nb = N / R;
  constexpr int twstep = N / L;
  const int total = ntrans * nb;
  const int es = m * estride;
  for (int it = tid; it < total; it += nthr) {
    int t, bf;
    if constexpr (LOG2T >= 0) {
      bf = it >> LOG2T;
      t = it & ((1 << LOG2T) - 1);
    } else if constexpr (LOG2T == -2) {
      bf = it / ntrans;
      t = it - bf * ntrans;
    } else {
      t = it / nb;
      bf = it - t * nb;
    }
    const int blk = bf / m;
    const int j2 = bf - blk * m;
    float2* base = buf + t * tstride + (blk * L + j2) * estride;
    float2 x[R];
#pragma unroll
    for (int j = 0; j < R; ++j) x[j] = base[j * es];
    if constexpr (INV) {
#pragma unroll
      for (int k = 1; k < R; ++k) x[k] = cmul(x[k], cconj(__ldg(&tw[twstep * j2 * k])));
      dft_small<R, true>(x);
    } else {
      dft_small<R, false>(x);
#pragma unroll
      for (int k = 1; k < R; ++k) x[k] = cmul(x[k], __ldg(&tw[twstep * j2 * k]));
    }
#pragma unroll
    for (int j = 0; j < R; ++j) base[j * es] = x[j];
  }
}

template <int N, bool INV, int LOG2T, int SI = 0>
__device__ __forceinline__ void fixed_stages(float2* buf, int ntrans, int tstride, int estride,
                                             const float2* __restrict__ tw, int tid, int nthr) {
  if constexpr (SI < FixedFft<N>::count) {
    constexpr int S = INV ? (FixedFft<N>::count - 1 - SI) : SI;
    fixed_stage<N, FixedFft<N>::r[S], fixed_L<N, S>(), INV, LOG2T>(buf, ntrans, tstride, estride, tw, tid, nthr);
    __syncthreads();
    fixed_stages<N, INV, LOG2T, SI + 1>(buf, ntrans, tstride, estride, tw, tid, nthr);
  }
}

// Batched in-place transform with a compile-time plan (same contract as
// fft_smem).  LOG2T >= 0: columns, ntrans == 2^LOG2T; LOG2T == -2: columns,
// any ntrans; LOG2T == -1: rows (estride 1).
template <int N, bool INV, int LOG2T = -1>
__device__ __forceinline__ void fft_fixed(float2* buf, int ntrans, int tstride, int estride,
                                          const float2* __restrict__ tw) {
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nthr = blockDim.x * blockDim.y * blockDim.z;
  fixed_stages<N, INV, LOG2T>(buf, ntrans, tstride, estride, tw, tid, nthr);
}

// Dispatch helpers: NF > 0 uses the compile-time plan of length NF, NF == 0
// the runtime plan.
template <int NF, bool INV, int LOG2T = -1>
__device__ __forceinline__ void fft_any(float2* buf, int ntrans, int tstride, int estride, const FftPlan& p) {
  if constexpr (NF > 0) {
    fft_fixed<NF, INV, LOG2T>(buf, ntrans, tstride, estride, p.tw);
  } else {
    fft_smem<INV>(buf, ntrans, tstride, estride, p);
  }
}

// Column transforms with a column-resident thread mapping: thread tid keeps
// column t = tid % ntrans and walks the butterflies g, g + groups, ... of each
// stage (g = tid / ntrans, groups = nthr / ntrans), so the index arithmetic
// is one division per call instead of one per butterfly, and a warp touches
// neighbouring columns of one butterfly.  Needs ntrans <= nthr (callers fall
// back to fft_fixed otherwise).
template <int N, int R, int L, bool INV>
__device__ __forceinline__ void fixed_col_stage(float2* buf, int stride, const float2* __restrict__ tw, int t, int g,
                                                int groups) {
  constexpr int m = L / R;
  constexpr int nb = N / R;
  constexpr int twstep = N / L;
  if (g >= groups) return;
  const size_t es = (size_t)m * stride;
  for (int bf = g; bf < nb; bf += groups) {
    const int blk = bf / m, j2 = bf - blk * m;
    float2* base = buf + t + (size_t)(blk * L + j2) * stride;
    float2 x[R];
#pragma unroll
    for (int j = 0; j < R; ++j) x[j] = base[j * es];
    if constexpr (INV) {
#pragma unroll
      for (int k = 1; k < R; ++k) x[k] = cmul(x[k], cconj(__ldg(&tw[twstep * j2 * k])));
      dft_small<R, true>(x);
    } else {
      dft_small<R, false>(x);
#pragma unroll
      for (int k = 1; k < R; ++k) x[k] = cmul(x[k], __ldg(&tw[twstep * j2 * k]));
    }
#pragma unroll
    for (int j = 0; j < R; ++j) base[j * es] = x[j];
  }
}

template <int N, bool INV, int SI = 0>
__device__ __forceinline__ void fixed_col_stages(float2* buf, int stride, const float2* __restrict__ tw, int t, int g,
                                                 int groups) {
  if constexpr (SI < FixedFft<N>::count) {
    constexpr int S = INV ? (FixedFft<N>::count - 1 - SI) : SI;
    fixed_col_stage<N, FixedFft<N>::r[S], fixed_L<N, S>(), INV>(buf, stride, tw, t, g, groups);
    __syncthreads();
    fixed_col_stages<N, INV, SI + 1>(buf, stride, tw, t, g, groups);
  }
}

// Columns t < ntrans of a [N][stride] buffer (element i of column t at
// buf[t + i * stride]).  Caller synchronises before; ends with __syncthreads().
template <int NF, bool INV>
__device__ __forceinline__ void fft_any_cols(float2* buf, int ntrans, int stride, const FftPlan& p) {
  const int nthr = blockDim.x;
  if constexpr (NF > 0) {
    if (ntrans <= nthr) {
      const int tid = threadIdx.x;
      fixed_col_stages<NF, INV>(buf, stride, p.tw, tid % ntrans, tid / ntrans, nthr / ntrans);
      return;
    }
  }
  fft_any<NF, INV, -2>(buf, ntrans, 1, stride, p);
}


template <int NF>
__device__ __forceinline__ int freq2pos(int k, const FftPlan& p) {
  if constexpr (NF > 0) {
    return fixed_freq2pos<NF>(k);
  } else {
    return fft_freq2pos(k, p);
  }
}

template <int NF>
__device__ __forceinline__ int pos2freq(int pos, const FftPlan& p) {
  if constexpr (NF > 0) {
    return fixed_pos2freq<NF>(pos);
  } else {
    return fft_pos2freq(pos, p);
  }
}

// Host dispatch of a kernel template on the transform length.
#define PHGPU_DISPATCH_N(n, ...)            \
  switch (n) {                              \
    case 64: {                              \
      constexpr int NF = 64;                \
      __VA_ARGS__;                          \
    } break;                                \
    case 128: {                             \
      constexpr int NF = 128;               \
      __VA_ARGS__;                          \
    } break;                                \
    case 200: {                             \
      constexpr int NF = 200;               \
      __VA_ARGS__;                          \
    } break;                                \
    case 256: {                             \
      constexpr int NF = 256;               \
      __VA_ARGS__;                          \
    } break;                                \
    case 512: {                             \
      constexpr int NF = 512;               \
      __VA_ARGS__;                          \
    } break;                                \
    case 320: {                             \
      constexpr int NF = 320;               \
      __VA_ARGS__;                          \
    } break;                                \
    default: {                              \
      constexpr int NF = 0;                 \
      __VA_ARGS__;                          \
    } break;                                \
  }

}  // namespace phgpu
