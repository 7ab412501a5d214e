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

// Packed FP32 pairs (sm_100 FADD2 / FFMA2 / FMUL2, PK = true): one
// instruction for both components of a complex sum, or of a complex times a
// real constant; PK = false gives the same arithmetic per component.  The
// rotations by +-i swap the components, which a packed pair cannot do for
// free, so the sums that take them stay per component.
template <bool PK>
__device__ __forceinline__ float2 padd(float2 a, float2 b) {
  if constexpr (PK) return __fadd2_rn(a, b);
  else return make_float2(a.x + b.x, a.y + b.y);
}
template <bool PK>
__device__ __forceinline__ float2 psub(float2 a, float2 b) {
  if constexpr (PK) return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a);
  else return make_float2(a.x - b.x, a.y - b.y);
}
// c + s a
template <bool PK>
__device__ __forceinline__ float2 pfma(float s, float2 a, float2 c) {
  if constexpr (PK) return __ffma2_rn(make_float2(s, s), a, c);
  else return make_float2(__fmaf_rn(s, a.x, c.x), __fmaf_rn(s, a.y, c.y));
}
template <bool PK>
__device__ __forceinline__ float2 pmul(float s, float2 a) {
  if constexpr (PK) return __fmul2_rn(make_float2(s, s), a);
  else return make_float2(s * a.x, s * a.y);
}
// a + i*sg*d and a - i*sg*d
template <bool INV>
__device__ __forceinline__ void rot_pm(float2 a, float2 d, float2& plus, float2& minus) {
  if constexpr (INV) {  // sg = +1: i d = (-d.y, d.x)
    plus = make_float2(a.x - d.y, a.y + d.x);
    minus = make_float2(a.x + d.y, a.y - d.x);
  } else {  // sg = -1: -i d = (d.y, -d.x)
    plus = make_float2(a.x + d.y, a.y - d.x);
    minus = make_float2(a.x - d.y, a.y + d.x);
  }
}

template <int R, bool INV, bool PK = true>
__device__ __forceinline__ void dft_small(float2 (&x)[R]) {
  constexpr float sg = INV ? 1.0f : -1.0f;  // exponent sign
  if constexpr (R == 2) {
    const float2 a = x[0], b = x[1];
    x[0] = padd<PK>(a, b);
    x[1] = psub<PK>(a, b);
  } else if constexpr (R == 3) {
    const float s3 = 0.86602540378443864676f;
    const float2 t1 = padd<PK>(x[1], x[2]);
    const float2 t2 = psub<PK>(x[1], x[2]);
    const float2 y0 = padd<PK>(x[0], t1);
    const float2 m1 = pfma<PK>(-0.5f, t1, x[0]);
    // m1 +- i*sg*s3*t2
    rot_pm<INV>(m1, pmul<PK>(s3, t2), x[1], x[2]);
    x[0] = y0;
  } else if constexpr (R == 4) {
    const float2 t0 = padd<PK>(x[0], x[2]);
    const float2 t1 = psub<PK>(x[0], x[2]);
    const float2 t2 = padd<PK>(x[1], x[3]);
    const float2 d = psub<PK>(x[1], x[3]);
    x[0] = padd<PK>(t0, t2);
    x[2] = psub<PK>(t0, t2);
    rot_pm<INV>(t1, d, x[1], x[3]);
  } else if constexpr (R == 5) {
    const float c1 = 0.30901699437494742410f, c2 = -0.80901699437494742410f;
    const float s1 = 0.95105651629515357212f, s2 = 0.58778525229247312917f;
    const float2 t1 = padd<PK>(x[1], x[4]), t2 = padd<PK>(x[2], x[3]);
    const float2 t3 = psub<PK>(x[1], x[4]), t4 = psub<PK>(x[2], x[3]);
    const float2 y0 = padd<PK>(x[0], padd<PK>(t1, t2));
    const float2 a1 = pfma<PK>(c2, t2, pfma<PK>(c1, t1, x[0]));
    const float2 a2 = pfma<PK>(c1, t2, pfma<PK>(c2, t1, x[0]));
    const float2 b1 = pfma<PK>(s2, t4, pmul<PK>(s1, t3));
    const float2 b2 = pfma<PK>(-s1, t4, pmul<PK>(s2, t3));
    // y1 = a1 + i*sg*b1, y4 = a1 - i*sg*b1, y2 = a2 + i*sg*b2, y3 = a2 - i*sg*b2
    x[0] = y0;
    rot_pm<INV>(a1, b1, x[1], x[4]);
    rot_pm<INV>(a2, b2, x[2], x[3]);
  } else if constexpr (R == 8) {
    float2 e[4] = {x[0], x[2], x[4], x[6]};
    float2 o[4] = {x[1], x[3], x[5], x[7]};
    dft_small<4, INV, PK>(e);
    dft_small<4, INV, PK>(o);
    const float h = 0.70710678118654752440f;
    // w8^k = exp(sg * i * pi k / 4): o1 w8 = h (o.x - sg o.y, o.y + sg o.x),
    // o3 w8^3 = (-h (o.x + sg o.y), h (sg o.x - o.y))
    const float2 o1 = pmul<PK>(h, make_float2(o[1].x - sg * o[1].y, o[1].y + sg * o[1].x));
    const float2 p3 = make_float2(o[3].x + sg * o[3].y, sg * o[3].x - o[3].y);
    const float2 o3 = PK ? __fmul2_rn(make_float2(-h, h), p3) : make_float2(-h * p3.x, h * p3.y);
    x[0] = padd<PK>(e[0], o[0]);
    x[4] = psub<PK>(e[0], o[0]);
    x[1] = padd<PK>(e[1], o1);
    x[5] = psub<PK>(e[1], o1);
    rot_pm<INV>(e[2], o[2], x[2], x[6]);
    x[3] = padd<PK>(e[3], o3);
    x[7] = psub<PK>(e[3], o3);
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
    // m == 1: j2 == 0, every twiddle is 1 (a block-uniform branch)
    if (INV) {
      if (m > 1) {
#pragma unroll
        for (int k = 1; k < R; ++k) x[k] = cmul(x[k], cconj(__ldg(&tw[twstep * j2 * k])));
      }
      dft_small<R, true>(x);
    } else {
      dft_small<R, false>(x);
      if (m > 1) {
#pragma unroll
        for (int k = 1; k < R; ++k) x[k] = cmul(x[k], __ldg(&tw[twstep * j2 * k]));
      }
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
      dft_small<R, true, false>(x);
    } else {
      dft_small<R, false, false>(x);
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
// PODD: element i of a column sits `podd` further when i is odd (a row-parity
// slot that spreads neighbouring rows over both halves of the banks).
template <int N, int R, int L, bool INV, bool PODD = false>
__device__ __forceinline__ void fixed_col_stage(float2* buf, int stride, const float2* __restrict__ tw, int t, int g,
                                                int groups, int podd = 0) {
  constexpr int m = L / R;
  constexpr int nb = N / R;
  constexpr int twstep = N / L;
  if (g >= groups) return;
  const size_t es = (size_t)m * stride;
  for (int bf = g; bf < nb; bf += groups) {
    const int blk = bf / m, j2 = bf - blk * m;
    const int r0 = blk * L + j2;
    float2* base = buf + t + (size_t)r0 * stride;
    // element j is row r0 + j m: its parity is r0's when j m is even
    const int po0 = PODD ? (r0 & 1) * podd : 0, po1 = PODD ? podd - po0 : 0;
    float2 x[R];
#pragma unroll
    for (int j = 0; j < R; ++j) x[j] = base[j * es + (((j * m) & 1) ? po1 : po0)];
    // m == 1 (the last forward / first inverse stage): j2 == 0, every twiddle is 1
    if constexpr (INV) {
      if constexpr (m > 1) {
#pragma unroll
        for (int k = 1; k < R; ++k) x[k] = cmul(x[k], cconj(__ldg(&tw[twstep * j2 * k])));
      }
      dft_small<R, true>(x);
    } else {
      dft_small<R, false>(x);
      if constexpr (m > 1) {
#pragma unroll
        for (int k = 1; k < R; ++k) x[k] = cmul(x[k], __ldg(&tw[twstep * j2 * k]));
      }
    }
#pragma unroll
    for (int j = 0; j < R; ++j) base[j * es + (((j * m) & 1) ? po1 : po0)] = x[j];
  }
}

template <int N, bool INV, bool PODD = false, int SI = 0>
__device__ __forceinline__ void fixed_col_stages(float2* buf, int stride, const float2* __restrict__ tw, int t, int g,
                                                 int groups, int podd = 0) {
  if constexpr (SI < FixedFft<N>::count) {
    constexpr int S = INV ? (FixedFft<N>::count - 1 - SI) : SI;
    fixed_col_stage<N, FixedFft<N>::r[S], fixed_L<N, S>(), INV, PODD>(buf, stride, tw, t, g, groups, podd);
    __syncthreads();
    fixed_col_stages<N, INV, PODD, SI + 1>(buf, stride, tw, t, g, groups, podd);
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

// The same with the row-parity slot: element i of column t at
// buf[t + i * stride + (i odd ? podd : 0)].  Compile-time lengths only, and
// ntrans <= blockDim.x.
template <int NF, bool INV>
__device__ __forceinline__ void fft_fixed_cols_podd(float2* buf, int ntrans, int stride, int podd,
                                                    const float2* __restrict__ tw) {
  static_assert(NF > 0, "row-parity slots need a compile-time plan");
  const int tid = threadIdx.x, nthr = blockDim.x;
  fixed_col_stages<NF, INV, true>(buf, stride, tw, tid % ntrans, tid / ntrans, nthr / ntrans, podd);
}


// Column transforms with every count known at compile time: NTRANS columns
// of a buffer with row stride STRIDE, NTHR threads (== blockDim.x), so the
// shared-memory offsets and the thread-to-column split fold to constants.
// PODD as in fixed_col_stage.
template <int NF, bool INV, int NTRANS, int STRIDE, int NTHR, bool PODD>
__device__ __forceinline__ void fixed_cols_ct(float2* buf, const float2* __restrict__ tw, int podd) {
  static_assert(NF > 0 && NTRANS <= NTHR, "compile-time column plan");
  const int tid = threadIdx.x;
  fixed_col_stages<NF, INV, PODD>(buf, STRIDE, tw, tid % NTRANS, tid / NTRANS, NTHR / NTRANS, podd);
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
