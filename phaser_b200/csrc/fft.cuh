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
      default: break;
    }
    __syncthreads();
  }
}

}  // namespace phgpu
