// Zero-padded translation correlation (spatial zero padding p > 0).
//
// Reference behaviour (SpatialCorrelation, phaser_core/src/backend/
// correlation/spatial-correlation.cc:11-45,78-83,142-161,223-230, and its
// Laplace / low-pass subclasses, spatial-correlation-laplace.cc:17-50,
// spatial-correlation-low-pass.cc:40-69), with M = N + 2p:
//   * each channel's r2c_3d at N fills the first V = N^2 (N/2 + 1) entries of
//     an N^3-long buffer (F_ / G_, zero at construction);
//   * Laplace and low-pass FFT-shift the whole N^3 buffer (std::rotate), so
//     the shifted entries whose source lies in [V, N^3) carry what the buffer
//     held there: the previous channel's shifted spectrum, which is the
//     previous channel's r2c output at source - (N^3 - mid); for the first
//     channel that is the previous call's last channel (zero before the
//     first call);
//   * Laplace fuses the channels positionally on the shifted index (the same
//     rule as the unpadded path, zero channels included with their tails);
//   * the product C = F conj(G) of linear index idx (all of [0, N^3), or the
//     low-pass cube) goes to computeZeroPaddedIndex(idx) = Sub2Ind(i + p,
//     j + p, k + p, M, M) with (i, j, k) = Ind2Sub(idx, N, N);
//   * Laplace and low-pass IFFT-shift the first N^3 entries of the M^3
//     buffer; c2r_3d at M reads its first M^2 (M/2 + 1) entries as a half
//     spectrum [kz][kx][ky]; every other entry is zero (the reference zeroes
//     the product buffer after each inverse).
// The low-pass class never clears its product buffer and FFTW's c2r leaves
// that buffer's contents algorithm-specific, so only its first call on a
// fresh object is defined: mode 2 reproduces that call (zero tails).
//
// GPU passes: the unpadded forward (r2c along y, FFT along x) is reused; a z
// pass completes the 3-D spectra; one thread per linear index gathers the
// channel values, fuses, multiplies and scatters into the padded half
// spectrum (z at its digit-reversed position for the inverse); an inverse z
// pass at M; the unpadded inverse kernels (x inverse, c2r along y, argmax)
// at M.  The padded path is not performance-tuned: the reference's run
// scripts leave spatial padding at 0.
#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.h"

namespace phgpu {
namespace {

constexpr int kPadZThreads = 256;
constexpr int kPadZCols = 8;

// z transform of kPadZCols ky columns at one x of one array.
template <bool INV>
__global__ void __launch_bounds__(kPadZThreads) k_pad_zfft(float2* __restrict__ base, size_t array_stride, int n,
                                                           int nx, int H, int H2p, FftPlan plan) {
  extern __shared__ float2 buf[];  // [n][kPadZCols]
  const int ky0 = blockIdx.x * kPadZCols;
  const int x = blockIdx.y;
  float2* arr = base + (size_t)blockIdx.z * array_stride;
  for (int e = threadIdx.x; e < n * kPadZCols; e += blockDim.x) {
    const int z = e / kPadZCols, w = e - z * kPadZCols;
    const int ky = ky0 + w;
    buf[e] = ky < H ? arr[((size_t)z * nx + x) * H2p + ky] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  fft_smem<INV>(buf, kPadZCols, 1, kPadZCols, plan);
  for (int e = threadIdx.x; e < n * kPadZCols; e += blockDim.x) {
    const int z = e / kPadZCols, w = e - z * kPadZCols;
    const int ky = ky0 + w;
    if (ky < H) arr[((size_t)z * nx + x) * H2p + ky] = buf[e];
  }
}

// Value of a full N-sized spectrum at FFTW half-spectrum index `flat`.
__device__ __forceinline__ float2 spec_at(const float2* __restrict__ arr, uint32_t flat, const PadArgs& a) {
  const uint32_t N = (uint32_t)a.N, H = N / 2 + 1;
  const uint32_t kz = flat / (N * H), rem = flat - kz * N * H;
  const uint32_t kx = rem / H, ky = rem - kx * H;
  const int zp = fft_freq2pos((int)kz, a.planN);
  const int xp = a.x_natural_N ? (int)kx : fft_freq2pos((int)kx, a.planN);
  return arr[((size_t)zp * N + (size_t)xp) * spatial_h2p(a.N) + ky];
}

__global__ void __launch_bounds__(256) k_pad_fuse(PadArgs a) {
  const uint32_t N = (uint32_t)a.N, M = (uint32_t)a.M, p = (uint32_t)a.pad;
  const uint32_t nv = N * N * N;
  const uint32_t V = N * N * (N / 2 + 1);
  const uint32_t mid = (nv & 1u) ? (nv >> 1) + 1u : (nv >> 1);  // FFTShift rotation
  const size_t plane = (size_t)N * N * spatial_h2p(a.N);
  const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nv) return;
  const uint32_t j = idx % N, i = (idx / N) % N, k = idx / (N * N);
  if (a.mode == 2 && (i < a.lp_lo || i > a.lp_hi || j < a.lp_lo || j > a.lp_hi || k < a.lp_lo || k > a.lp_hi))
    return;
  float2 F, G;
  if (a.mode == 0) {
    // no shift; the buffer tail past V stays zero
    const float2* sf = a.spec + (size_t)a.first_ch * plane;
    const float2* sg = a.spec + (size_t)(a.spec_ch + a.first_ch) * plane;
    F = idx < V ? spec_at(sf, idx, a) : make_float2(0.f, 0.f);
    G = idx < V ? spec_at(sg, idx, a) : make_float2(0.f, 0.f);
  } else {
    uint32_t src = idx + mid;
    if (src >= nv) src -= nv;
    if (a.mode == 2) {
      // fresh object: the tail is zero
      const float2* sf = a.spec + (size_t)a.first_ch * plane;
      const float2* sg = a.spec + (size_t)(a.spec_ch + a.first_ch) * plane;
      F = src < V ? spec_at(sf, src, a) : make_float2(0.f, 0.f);
      G = src < V ? spec_at(sg, src, a) : make_float2(0.f, 0.f);
    } else {
      const bool tail = src >= V;
      const uint32_t flat = tail ? src + mid - nv : src;  // source in the previous channel for the tail
      const int op = fusion_op(idx, a.bands);
      float2 sf = make_float2(0.f, 0.f), sg = sf, mf = sf, mg = sf;
      float bf = -1.f, bg = -1.f;
      for (int c = 0; c < a.n_ch; ++c) {
        // which spectrum holds this channel's value at idx
        const int owner = tail ? c - 1 : c;
        float2 u = make_float2(0.f, 0.f), v = u;
        if (owner >= 0 && owner < a.n_spec) {
          u = spec_at(a.spec + (size_t)owner * plane, flat, a);
          v = spec_at(a.spec + (size_t)(a.spec_ch + owner) * plane, flat, a);
        } else if (owner < 0) {
          if (a.prev_f) u = spec_at(a.prev_f, flat, a);
          if (a.prev_g) v = spec_at(a.prev_g, flat, a);
        }
        sf = cadd(sf, u);
        sg = cadd(sg, v);
        const float eu = u.x * u.x + u.y * u.y;
        const float ev = v.x * v.x + v.y * v.y;
        mf = eu > bf ? u : mf;
        bf = eu > bf ? eu : bf;
        mg = ev > bg ? v : mg;
        bg = ev > bg ? ev : bg;
      }
      const float inv = a.inv_total;
      F = op == kFuseMax ? mf : (op == kFuseMean ? make_float2(sf.x * inv, sf.y * inv) : make_float2(0.f, 0.f));
      G = op == kFuseMax ? mg : (op == kFuseMean ? make_float2(sg.x * inv, sg.y * inv) : make_float2(0.f, 0.f));
    }
  }
  const float2 c = make_float2(F.x * G.x - F.y * (-G.y), F.x * (-G.y) + F.y * G.x);
  // computeZeroPaddedIndex, then the IFFT shift of the first N^3 entries
  uint32_t y = (i + p) * M + (j + p) + M * M * (k + p);
  if (a.mode != 0 && y < nv) {
    y += nv - (nv >> 1);
    if (y >= nv) y -= nv;
  }
  const uint32_t HM = M / 2 + 1;
  if (y >= M * M * HM) return;  // beyond the half spectrum the c2r reads
  const uint32_t kz = y / (M * HM), rem = y - kz * M * HM;
  const uint32_t kx = rem / HM, ky = rem - kx * HM;
  const int zp = fft_freq2pos((int)kz, a.planM);
  const int xp = a.x_natural_M ? (int)kx : fft_freq2pos((int)kx, a.planM);
  a.cspec[((size_t)zp * M + (size_t)xp) * spatial_h2p(a.M) + ky] = c;
}

}  // namespace

cudaError_t launch_pad_zfft(float2* base, size_t array_stride, int n_arrays, int n, int nx, int H, int inverse,
                            const FftPlan& plan, cudaStream_t st) {
  const size_t sm = (size_t)n * kPadZCols * sizeof(float2);
  dim3 g((H + kPadZCols - 1) / kPadZCols, nx, n_arrays);
  const int H2p = spatial_h2p(n);
  if (sm > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_pad_zfft<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_pad_zfft<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
  }
  if (inverse)
    k_pad_zfft<true><<<g, kPadZThreads, sm, st>>>(base, array_stride, n, nx, H, H2p, plan);
  else
    k_pad_zfft<false><<<g, kPadZThreads, sm, st>>>(base, array_stride, n, nx, H, H2p, plan);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_pad_fuse(const PadArgs& a, cudaStream_t st) {
  const uint32_t nv = (uint32_t)a.N * (uint32_t)a.N * (uint32_t)a.N;
  k_pad_fuse<<<(nv + 255) / 256, 256, 0, st>>>(a);
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace phgpu
