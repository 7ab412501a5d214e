// Translation stage: voxelisation, 3-D real FFTs, fused cross power, inverse
// real FFT and argmax.
//
// Reference behaviour:
//  * PhaseAligner::discretizePointcloud (phaser_core/src/backend/alignment/
//    phase-aligner.cc:71-131) with igl::histc (phaser_core/include/igl/
//    histc.cpp:34-73): float edges, binary search, -1 for out-of-range
//    coordinates, lin = uint32(bx)*N + uint32(by) + N*N*uint32(bz) with uint32
//    wrap-around and the `lin > N^3` guard; per-voxel means of intensity,
//    range (sqrtf of the float squared norm), reflectivity, ambient; empty
//    voxels 0.  Channel order {intensity, range, reflectivity, ambient}.
//  * SpatialCorrelationLaplace::correlateSignals (phaser_core/src/backend/
//    correlation/spatial-correlation-laplace.cc:17-89) with
//    SpatialCorrelation::complexMulSeq / c2r (spatial-correlation.cc:52-161):
//    r2c_3d over [z][x][y] (y halved), positional pyramid fusion on the
//    FFT-shifted linear index of the N*N*(N/2+1) half spectrum, C = F conj(G),
//    unnormalised c2r_3d (complex inverse over z and x, then the real
//    half-complex inverse over y, which reads only the real part of the DC and
//    Nyquist terms), first-occurrence argmax of the signed output.
//
// Passes (FP32): A1 r2c along y per row; A2 forward FFT along x per (z, ky
// tile); B forward FFT along z for all channels of both clouds per (x, ky
// tile) + fusion + cross power + inverse FFT along z; C1 inverse FFT along x;
// C2 complex-to-real along y with argmax.  Forward transforms leave x and z in
// digit-reversed order; the inverse transforms consume that order directly.
#include <cuda.h>  // CUtensorMap (encoded through the runtime's driver entry point)

#include "fft2.cuh"
#include "kernels.h"

namespace phgpu {

// histc's bin (igl/histc.cpp:34-73): -1 outside [E[0], E[N-1]], else the
// result of its binary search over the sorted edges -- the largest l <= N-2
// with E[l] <= x, or N-1 when x == E[N-1] (NaN: N-2, where the search ends;
// N = 1: 0).
// The search is replaced by a start at the linear estimate (x - E[0]) * inv,
// inv = (N-1) / (E[N-1] - E[0]), corrected by exact comparisons with the
// edges, which gives the same bin in one or two loads instead of log2 N.
__device__ __forceinline__ int histc_bin(float x, const float* __restrict__ E, int N, float e0, float e1,
                                         float inv) {
  if (x < e0 || x > e1) return -1;
  if (N < 2) return 0;
  if (x != x) return N - 2;
  int l = (int)((x - e0) * inv);
  l = min(max(l, 0), N - 2);
  while (l > 0 && x < E[l]) --l;
  while (l < N - 2 && x >= E[l + 1]) ++l;
  return (x == E[l + 1]) ? l + 1 : l;
}

__global__ void k_voxelize(VoxelArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int np = a.n_dev ? (int)*a.n_dev : a.n_points;
  if (i >= np) return;
  const float4 p = a.xyzi[i];
  float x = p.x, y = p.y, z = p.z;
  if (a.has_T || a.T_dev) {
    // PCL 1.8 transformPointCloud order ((T0 x + T1 y) + T2 z) + T3
    float Tl[12];
    if (a.T_dev) {
#pragma unroll
      for (int k = 0; k < 12; ++k) Tl[k] = __ldg(&a.T_dev[k]);
    } else {
#pragma unroll
      for (int k = 0; k < 12; ++k) Tl[k] = a.T[k];
    }
    const float* T = Tl;
    const float nx = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(T[0], x), __fmul_rn(T[1], y)), __fmul_rn(T[2], z)), T[3]);
    const float ny = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(T[4], x), __fmul_rn(T[5], y)), __fmul_rn(T[6], z)), T[7]);
    const float nz = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(T[8], x), __fmul_rn(T[9], y)), __fmul_rn(T[10], z)), T[11]);
    x = nx;
    y = ny;
    z = nz;
  }
  const uint32_t N = (uint32_t)a.N;
  const float e0 = __ldg(&a.edges[0]), e1 = __ldg(&a.edges[a.N - 1]);
  const float inv = a.N > 1 ? (float)(a.N - 1) / (e1 - e0) : 0.0f;
  const uint32_t bx = (uint32_t)histc_bin(x, a.edges, a.N, e0, e1, inv);
  const uint32_t by = (uint32_t)histc_bin(y, a.edges, a.N, e0, e1, inv);
  const uint32_t bz = (uint32_t)histc_bin(z, a.edges, a.N, e0, e1, inv);
  const uint32_t lin = (bx * N + by) + (N * N * bz);
  const uint32_t nv = N * N * N;
  const bool ok = lin < nv;
  if (a.lin_out) a.lin_out[i] = ok ? lin : 0xffffffffu;
  if (!ok) return;
  // the row of lin, not (bz, bx): an out-of-range bin (-1) wraps into another row
  if (a.rowlive) a.rowlive[lin / N] = 1;
  float* g = a.grids;
  atomicAdd(&g[lin], p.w);
  const float r = sqrtf(__fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z)));
  atomicAdd(&g[(size_t)nv + lin], r);
  if (a.n_data_ch > 2) atomicAdd(&g[(size_t)2 * nv + lin], a.refl ? a.refl[i] : 0.0f);
  if (a.n_data_ch > 3) atomicAdd(&g[(size_t)3 * nv + lin], a.amb ? a.amb[i] : 0.0f);
  atomicAdd(&g[(size_t)a.n_data_ch * nv + lin], 1.0f);
}

cudaError_t launch_voxelize(const VoxelArgs& a, cudaStream_t st) {
  if (a.n_points > 0) {
    k_voxelize<<<(a.n_points + 255) / 256, 256, 0, st>>>(a);
    count_launches(1);
  }
  return cudaGetLastError();
}

__global__ void k_clear_voxels(const uint32_t* __restrict__ lin, int n_points, float* __restrict__ grids, size_t nv,
                               int n_planes, uint8_t* __restrict__ rowlive, int N, const uint32_t* __restrict__ n_dev) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (n_dev ? (int)*n_dev : n_points)) return;
  const uint32_t l = lin[i];
  if (l == 0xffffffffu) return;
  for (int p = 0; p < n_planes; ++p) grids[(size_t)p * nv + l] = 0.0f;
  if (rowlive) rowlive[l / (uint32_t)N] = 0;
}

cudaError_t launch_clear_voxels(const uint32_t* lin, int n_points, float* grids, size_t nv, int n_planes,
                                uint8_t* rowlive, int N, cudaStream_t st, const uint32_t* n_dev) {
  if (n_points > 0) {
    k_clear_voxels<<<(n_points + 255) / 256, 256, 0, st>>>(lin, n_points, grids, nv, n_planes, rowlive, N, n_dev);
    count_launches(1);
  }
  return cudaGetLastError();
}

// ---------------------------------------------------------------- A1
// mean of a voxel: sum / count, 0 for empty voxels (reference: non-finite -> 0)
__device__ __forceinline__ float voxel_mean(float v, float c) { return c > 0.0f ? v * __frcp_rn(c) : 0.0f; }

constexpr int kRowsR2C = 16;

// rows r = z*N + x of one channel; out spec[ch][r][ky], ky in [0, N/2].
// A block takes kRowsR2C rows; rows without any point (row flags of the
// voxeliser) are written as zeros without being read, and the live rows are
// transformed two at a time as the real and imaginary parts of one complex
// row, Z = X0 + i X1, separated afterwards by
//   X0[k] = (Z[k] + conj Z[-k]) / 2,   X1[k] = (Z[k] - conj Z[-k]) / 2i.
template <int NF>
__global__ void k_r2c_y(int N, const float* __restrict__ grid, const float* __restrict__ count,
                        const uint8_t* __restrict__ rowlive, float2* __restrict__ spec, FftPlan plan) {
  extern __shared__ float2 rows[];  // [kRowsR2C / 2][n] packed rows, then int pos[n]
  constexpr int R = kRowsR2C;
  __shared__ int s_slot[R];         // 2 * packed row + part, or -1 for a row without points
  __shared__ int s_src[R];          // live rows in order
  __shared__ int s_nlive;
  const int n = NF > 0 ? NF : N;
  const int H2 = n / 2 + 1;
  const int H2p = spatial_h2p(n);
  int* pos = reinterpret_cast<int*>(rows + (size_t)(R / 2) * n);
  const size_t nrows = (size_t)n * n;
  const size_t r0 = (size_t)blockIdx.x * R;
  if (threadIdx.x < 32) {
    const int rr = threadIdx.x;
    const bool live = rr < R && r0 + rr < nrows && (!rowlive || rowlive[r0 + rr]);
    const unsigned m = __ballot_sync(0xffffffffu, live);
    const int k = __popc(m & ((1u << rr) - 1u));
    if (rr < R) s_slot[rr] = live ? k : -1;
    if (live) s_src[k] = rr;
    if (rr == 0) s_nlive = __popc(m);
  }
  for (int k = threadIdx.x; k < n; k += blockDim.x) pos[k] = freq2pos<NF>(k, plan);
  __syncthreads();
  const int nlive = s_nlive;
  const int npk = (nlive + 1) / 2;
  for (int e = threadIdx.x; e < npk * n; e += blockDim.x) {
    const int pk = e / n, y = e - pk * n;
    float v[2] = {0.f, 0.f};
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int li = 2 * pk + h;
      if (li < nlive) {
        const size_t idx = (r0 + s_src[li]) * n + y;
        v[h] = count ? voxel_mean(grid[idx], count[idx]) : grid[idx];
      }
    }
    rows[e] = make_float2(v[0], v[1]);
  }
  __syncthreads();
  if (npk > 0) fft_any<NF, false>(rows, npk, n, 1, plan);
  for (int e = threadIdx.x; e < R * H2; e += blockDim.x) {
    const int rr = e / H2, ky = e - rr * H2;
    const size_t r = r0 + rr;
    if (r >= nrows) continue;
    const int sl = s_slot[rr];
    float2 X = make_float2(0.f, 0.f);
    if (sl >= 0) {
      const float2* Z = rows + (size_t)(sl >> 1) * n;
      const float2 a = Z[pos[ky]], b = Z[pos[ky == 0 ? 0 : n - ky]];
      X = (sl & 1) ? make_float2(0.5f * (a.y + b.y), -0.5f * (a.x - b.x))  // (a - conj b) / 2i
                   : make_float2(0.5f * (a.x + b.x), 0.5f * (a.y - b.y));  // (a + conj b) / 2
    }
    spec[r * H2p + ky] = X;
  }
}

// ---------------------------------------------------------------- A2 / C1
// In-place transform along x for a tile of ky at one z: spec[z][x][ky].
template <int NF, bool INV>
__global__ void k_fft_x(int N, float2* __restrict__ spec, FftPlan plan) {
  extern __shared__ float2 tile[];
  constexpr int Wt = 16;
  const int n = NF > 0 ? NF : N;
  const int H2 = n / 2 + 1;
  const int H2p = spatial_h2p(n);
  const int ky0 = blockIdx.x * Wt;
  const int wt = min(Wt, H2 - ky0);
  float2* base = spec + (size_t)blockIdx.y * n * H2p;
  for (int e = threadIdx.x; e < n * Wt; e += blockDim.x) {
    const int x = e / Wt, t = e % Wt;
    tile[e] = t < wt ? base[(size_t)x * H2p + ky0 + t] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  fft_any<NF, INV, 4>(tile, Wt, 1, Wt, plan);
  for (int e = threadIdx.x; e < n * Wt; e += blockDim.x) {
    const int x = e / Wt, t = e % Wt;
    if (t < wt) base[(size_t)x * H2p + ky0 + t] = tile[e];
  }
}

// ---------------------------------------------------------------- B
// For one x position (digit-reversed) and a tile of ky: forward z FFT of all
// 2C arrays, fusion + cross power, inverse z FFT of the product.
//
// The [z][array][ky tile] block arrives by one bulk tensor copy per z chunk
// (TMA, when the host could encode the tensor map; each box <= 256 z rows)
// into the same layout the element loader produces.  Dynamic shared memory:
// tile [zrows][rowlen] float2 | mbarrier (16 B) | fusion bands.

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Waits for phase 0 of a shared-memory mbarrier; gives up after a bounded
// number of polls (returns false).
__device__ __forceinline__ bool mbar_wait0(uint64_t* bar) {
  uint32_t done = 0;
  for (int it = 0; it < (1 << 22) && !done; ++it) {
    asm volatile("{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0; selp.u32 %0, 1, 0, p; }"
                 : "=r"(done)
                 : "r"(smem_addr(bar))
                 : "memory");
  }
  return done != 0;
}

// Channel sums (MEAN) and the first channel of largest energy (MAX) of both
// sides at one position of a fuse_z tile row: channel c of side f in slot c,
// of side g in slot C + c.  Odd rows (odd = true) load g before f, which
// keeps the two loads on different banks (see k_fuse_z).  CC > 0: C == CC
// known at compile time.
template <int CC>
__device__ __forceinline__ void fuse_sides(const float2* row, int C, int Wt, int t, bool odd, float2& sf, float2& sg,
                                           float2& mf, float2& mg) {
  if constexpr (CC > 0) C = CC;
  sf = make_float2(0.f, 0.f);
  sg = sf;
  mf = sf;
  mg = sf;
  float bf = -1.f, bg = -1.f;
#pragma unroll
  for (int c = 0; c < (CC > 0 ? CC : C); ++c) {
    const float2 p0 = row[(odd ? C + c : c) * Wt + t];
    const float2 p1 = row[(odd ? c : C + c) * Wt + t];
    const float2 u = odd ? p1 : p0;
    const float2 v = odd ? p0 : p1;
    sf = cadd(sf, u);
    sg = cadd(sg, v);
    const float eu = u.x * u.x + u.y * u.y;
    const float ev = v.x * v.x + v.y * v.y;
    mf = eu > bf ? u : mf;
    bf = eu > bf ? eu : bf;
    mg = ev > bg ? v : mg;
    bg = ev > bg ? ev : bg;
  }
}

struct FuseZTma {
  int enabled;  // tensor map valid
  int zbox;     // z rows per copy
  int chunks;   // copies (zbox * chunks >= N)
};

// Two blocks per SM for the compile-time lengths (the bound lets the
// compiler schedule for it: 0.1294 against 0.1336 ms at N = 200; 640 or 672
// threads, whose radix passes divide more evenly, ran the same); the runtime
// plan's generic transform needs its 128 registers.
// CA, CW > 0: the Laplace fusion of C = CA / 2 channels with tile width CW,
// known at compile time (every shared-memory offset of the transforms folds
// to a constant); CA = CW = 0: any shape (the host picks).
constexpr int kFuseZThreads = 512;
template <int NF, int CA = 0, int CW = 0>
__global__ void __launch_bounds__(kFuseZThreads, NF > 0 ? 2 : 1)
    k_fuse_z(SpatialArgs a, FftPlan plan, int Wt_arg, int x_natural, const __grid_constant__ CUtensorMap tmap,
             FuseZTma tma) {
  extern __shared__ __align__(128) float2 tile[];  // [z][arr][t]
  static_assert(CA == 0 || (NF > 0 && CW == 8 && CA % 2 == 0), "compile-time shape: NF > 0, Wt = 8");
  const int N = NF > 0 ? NF : a.N;
  const int H2 = N / 2 + 1;
  const int H2p = spatial_h2p(N);
  const int C = CA > 0 ? CA / 2 : a.n_data_ch;
  const int A = CA > 0 ? CA : (a.laplace ? 2 * C : 2);
  const int Wt = CW > 0 ? CW : Wt_arg;
  const int ky0 = blockIdx.x * Wt;
  const int wt = min(Wt, H2 - ky0);
  const int xp = blockIdx.y;
  const size_t plane = (size_t)N * N * H2p;
  const int rowlen = A * Wt;
  const int zrows = tma.enabled ? tma.zbox * tma.chunks : N;
  uint64_t* bar = reinterpret_cast<uint64_t*>(tile + (size_t)zrows * rowlen);
  FusionBands* s_bands = reinterpret_cast<FusionBands*>(bar + 2);
  int* s_kz = reinterpret_cast<int*>(s_bands + 1);  // [N] z frequency of each position
  if (threadIdx.x == 0) *s_bands = a.bands;  // divergent band lookups are cheap in shared memory
  for (int zp = threadIdx.x; zp < N; zp += kFuseZThreads) s_kz[zp] = pos2freq<NF>(zp, plan);
  // the bulk copy needs a 128-byte aligned destination (block-uniform test)
  const bool use_tma = tma.enabled && (smem_addr(tile) & 127u) == 0;
  if (use_tma) {
    if (threadIdx.x == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)));
      asm volatile("fence.mbarrier_init.release.cluster;");
      asm volatile("fence.proxy.async.shared::cta;");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      const uint32_t bytes = (uint32_t)((size_t)zrows * rowlen * sizeof(float2));
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                   : "memory");
      for (int ch = 0; ch < tma.chunks; ++ch) {
        const int z0 = ch * tma.zbox;
        asm volatile(
            "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
            " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_addr(tile + (size_t)z0 * rowlen)),
            "l"(&tmap), "r"(ky0), "r"(0), "r"(xp), "r"(z0), "r"(smem_addr(bar))
            : "memory");
      }
    }
    if (!mbar_wait0(bar)) {
      if (threadIdx.x == 0) atomicOr(a.status, 1ull);
      mbar_wait0(bar);  // once more (bounded) so no copy is left in flight
    }
  } else {
    // tiles start at ky0 (multiple of Wt) in rows padded to 8 complex: load two
    // complex per 16-byte access
    const int half = Wt >> 1;
    for (int e = threadIdx.x; e < N * A * half; e += kFuseZThreads) {
      const int z = e / (A * half), rem = e - z * (A * half), ar = rem / half, t2 = rem - ar * half;
      // arrays: f channels 0..C-1 then g channels; plain mode uses channel 0 of
      // each side, the low-pass mode channel 1
      const int src = a.laplace ? ar : (ar == 0 ? a.lowpass : C + a.lowpass);
      const float4 v = *reinterpret_cast<const float4*>(
          a.spec + (size_t)src * plane + ((size_t)z * N + xp) * H2p + ky0 + 2 * t2);
      float2* d = tile + (size_t)z * rowlen + ar * Wt + 2 * t2;
      d[0] = make_float2(v.x, v.y);
      d[1] = make_float2(v.z, v.w);
    }
  }
  __syncthreads();
  if constexpr (CA > 0)
    fixed_cols_ct<NF, false, CA * CW, CA * CW, kFuseZThreads, false>(tile, plan.tw, 0);
  else
    fft_any_cols<NF, false>(tile, rowlen, rowlen, plan);
  const int kx = x_natural ? xp : pos2freq<NF>(xp, plan);
  const uint32_t nv = (uint32_t)N * (uint32_t)N * (uint32_t)N;
  // MEAN divides by the total channel count: a product with the reciprocal,
  // exact for the reference's 4 channels (within one rounding otherwise)
  const float inv_total = 1.0f / (float)a.n_total_ch;
  // Wt is a power of two (fuse_z_tile_ok): shifts, not a runtime division per element
  const int lwt = __ffs(Wt) - 1;
  // With Wt = 8 a half-warp covers two rows whose slots start on the same
  // banks (a row is A * 64 bytes): odd rows load their two sides in the
  // opposite order (conflict-free when the slots of a channel's sides are an
  // odd number of slots apart) and keep the product in slot 1 instead of 0,
  // which the inverse transform and the store follow.
  const int podd = (NF > 0 && Wt == 8) ? Wt : 0;
  for (int e = threadIdx.x; e < N * Wt; e += kFuseZThreads) {
    const int zp = e >> lwt, t = e & (Wt - 1);
    const bool odd = podd && (zp & 1);
    float2* row = tile + (size_t)zp * rowlen;
    float2 F, G;
    if (CA == 0 && !a.laplace) {
      const float2 p0 = row[(odd ? Wt : 0) + t], p1 = row[(odd ? 0 : Wt) + t];
      F = odd ? p1 : p0;
      G = odd ? p0 : p1;
      if (a.lowpass) {
        // keep the products whose FFT-shifted index p = (i N + j) + N^2 k has
        // i, j, k in [lp_lo, lp_hi]
        const int kz = s_kz[zp];
        const uint32_t klin = ((uint32_t)kz * N + (uint32_t)kx) * (uint32_t)H2 + (uint32_t)(ky0 + t);
        uint32_t p = klin + (nv >> 1);
        if (p >= nv || p < klin) p -= nv;
        const uint32_t n2 = (uint32_t)N * (uint32_t)N, kk = p / n2, rem = p - kk * n2;
        const uint32_t ii = rem / (uint32_t)N, jj = rem - ii * (uint32_t)N;
        if (ii < a.lp_lo || ii > a.lp_hi || jj < a.lp_lo || jj > a.lp_hi || kk < a.lp_lo || kk > a.lp_hi) {
          F = make_float2(0.f, 0.f);
          G = F;
        }
      }
    } else {
      const int kz = s_kz[zp];
      const uint32_t klin = ((uint32_t)kz * N + (uint32_t)kx) * (uint32_t)H2 + (uint32_t)(ky0 + t);
      // (klin + nv/2) mod nv with klin < nv
      uint32_t p = klin + (nv >> 1);
      if (p >= nv || p < klin) p -= nv;
      const int op = fusion_op(p, *s_bands);
      // one branch-free pass serves every rule (a divergent switch between
      // the rules cost more than the arithmetic): channel sums for MEAN, the
      // first channel of largest energy for MAX
      float2 sf, sg, mf, mg;
      if constexpr (CA > 0)
        fuse_sides<CA / 2>(row, C, Wt, t, odd, sf, sg, mf, mg);
      else if (C == 3)  // range, intensity, reflectivity: the loop unrolled
        fuse_sides<3>(row, 3, Wt, t, odd, sf, sg, mf, mg);
      else
        fuse_sides<0>(row, C, Wt, t, odd, sf, sg, mf, mg);
      const float inv = inv_total;
      F = op == kFuseMax ? mf : (op == kFuseMean ? make_float2(sf.x * inv, sf.y * inv) : make_float2(0.f, 0.f));
      G = op == kFuseMax ? mg : (op == kFuseMean ? make_float2(sg.x * inv, sg.y * inv) : make_float2(0.f, 0.f));
    }
    // complexMulSeq: C = F * conj(G); only this thread touches position (zp, t)
    row[(odd ? Wt : 0) + t] = make_float2(F.x * G.x - F.y * (-G.y), F.x * (-G.y) + F.y * G.x);
  }
  __syncthreads();
  if constexpr (CA > 0) {
    fixed_cols_ct<NF, true, CW, CA * CW, kFuseZThreads, true>(tile, plan.tw, CW);
  } else if constexpr (NF > 0) {
    if (podd)
      fft_fixed_cols_podd<NF, true>(tile, Wt, rowlen, podd, plan.tw);
    else
      fft_any_cols<NF, true>(tile, Wt, rowlen, plan);
  } else {
    fft_any_cols<NF, true>(tile, Wt, rowlen, plan);
  }
  for (int e = threadIdx.x; e < N * Wt; e += kFuseZThreads) {
    const int z = e >> lwt, t = e & (Wt - 1);
    if (t < wt) a.cspec[((size_t)z * N + xp) * H2p + ky0 + t] = tile[(size_t)z * rowlen + ((z & 1) ? podd : 0) + t];
  }
}

// ---------------------------------------------------------------- C2
// Real inverse over y of kRowsR2C rows with first-occurrence argmax.  A
// half-complex inverse reads only the real parts of the ky = 0 and ky = N/2
// terms, so each row is made exactly Hermitian that way, and rows are
// inverted two at a time as Z = X0 + i X1 (output x0 = Re, x1 = Im).
template <int NF>
__global__ void k_c2r_y(int N, const float2* __restrict__ cspec, FftPlan plan,
                        unsigned long long* __restrict__ argmax, float* __restrict__ volume, uint32_t limit) {
  extern __shared__ float2 rows[];  // [kRowsR2C / 2][n] packed rows, then int pos[n]
  constexpr int R = kRowsR2C;
  const int n = NF > 0 ? NF : N;
  const int H2 = n / 2 + 1;
  const int H2p = spatial_h2p(n);
  int* pos = reinterpret_cast<int*>(rows + (size_t)(R / 2) * n);
  const size_t nrows = (size_t)n * n;
  const size_t r0 = (size_t)blockIdx.x * R;
  for (int k = threadIdx.x; k < n; k += blockDim.x) pos[k] = freq2pos<NF>(k, plan);
  __syncthreads();
  const int hmax = (n - 1) / 2;  // last ky with a mirrored partner
  for (int e = threadIdx.x; e < (R / 2) * H2; e += blockDim.x) {
    const int pk = e / H2, ky = e - pk * H2;
    const size_t ra = r0 + 2 * pk, rb = ra + 1;
    float2 a = ra < nrows ? cspec[ra * H2p + ky] : make_float2(0.f, 0.f);
    float2 b = rb < nrows ? cspec[rb * H2p + ky] : make_float2(0.f, 0.f);
    if (ky == 0 || 2 * ky == n) {
      a.y = 0.f;
      b.y = 0.f;
    }
    float2* Z = rows + (size_t)pk * n;
    Z[pos[ky]] = make_float2(a.x - b.y, a.y + b.x);                                // a + i b
    if (ky >= 1 && ky <= hmax) Z[pos[n - ky]] = make_float2(a.x + b.y, b.x - a.y);  // conj a + i conj b
  }
  __syncthreads();
  fft_any<NF, true>(rows, R / 2, n, 1, plan);
  unsigned long long best = 0ull;
  for (int e = threadIdx.x; e < R * n; e += blockDim.x) {
    const int rr = e / n, y = e - rr * n;
    const size_t r = r0 + rr;
    if (r < nrows) {
      const float2 z = rows[(size_t)(rr >> 1) * n + y];
      const float v = (rr & 1) ? z.y : z.x;
      const uint32_t idx = (uint32_t)(r * n + y);
      const unsigned long long key = idx < limit ? pack_argmax(v, idx) : 0ull;
      best = key > best ? key : best;
      if (volume) volume[idx] = v;
    }
  }
  warp_argmax_commit(best, argmax);
}

// ---------------------------------------------------------------- z-slab
// Fused forward r2c over (x, y) of one z-slab of one channel (NF even, the
// slab of NF/2 x NF complex fits in shared memory).  Rows x = 2r and 2r+1 are
// packed as real and imaginary parts of one complex row; FFT over y (NF
// points), FFT over r (NF/2 points), then the two real spectra are separated
// in the 2-D frequency domain,
//   A = (W[ky][k] + conj W[-ky][-k]) / 2,  B = (W[ky][k] - conj W[-ky][-k]) / 2i,
// and combined over the even/odd x split,
//   X[k][ky] = A + w_N^k B,  X[k + N/2][ky] = A - w_N^k B.
// Output rows are in natural kx order.  Shared rows have the odd stride N + 1.


template <int NF>
__global__ void __launch_bounds__(tail_threads<NF>()) k_slab_fwd(const float* __restrict__ grids, size_t grid_cstride,
                                                   const float* __restrict__ count,
                                                   const uint8_t* __restrict__ rowlive, float2* __restrict__ spec,
                                                   size_t spec_cstride, FftPlan pN, FftPlan pH,
                                                   uint8_t* __restrict__ slab_nz) {
  constexpr int N = NF, NH = NF / 2, H2 = NF / 2 + 1, Q = NF / 4, S = NF + 1;
  constexpr int T = tail_threads<NF>();  // the launch's block size
  const int H2p = spatial_h2p(N);
  extern __shared__ float2 W[];  // [NH][S]
  __shared__ int s_flag[NH];      // packed row r may hold a point (row flags), else all zero
  __shared__ int s_live[NH];      // packed row r holds a non-zero value
  __shared__ int s_rows[NH];      // compact list of those rows
  __shared__ int s_nrows;
  __shared__ int s_posN[N], s_posH[NH];  // digit-reversed positions of frequencies
  const int z = blockIdx.x, c = blockIdx.y;
  const float* g = grids + (size_t)c * grid_cstride + (size_t)z * N * N;
  const float* cnt = count ? count + (size_t)z * N * N : nullptr;
  // slab_nz[c][z]: 0 when this slab of spectrum array c is known to hold zeros
  uint8_t* nz = slab_nz ? slab_nz + (size_t)c * N + z : nullptr;
  const int held_nonzero = nz ? *nz : 1;
  int any_flag = 0;
  for (int r = threadIdx.x; r < NH; r += T) {
    s_live[r] = 0;
    s_flag[r] = rowlive ? (rowlive[z * N + 2 * r] | rowlive[z * N + 2 * r + 1]) : 1;
    any_flag |= s_flag[r];
  }
  // a slab without a flagged row transforms to zero: nothing to do where the
  // array already holds zeros there (about half the slabs of a room scan, so
  // they leave before any other set-up)
  if (!__syncthreads_or(any_flag) && !held_nonzero) return;
  for (int r = threadIdx.x; r < NH; r += T) s_posH[r] = fixed_freq2pos<NH>(r);
  for (int k = threadIdx.x; k < N; k += T) s_posN[k] = fixed_freq2pos<N>(k);
  for (int e = threadIdx.x; e < NH * Q; e += T) {
    const int r = e / Q, y4 = (e - r * Q) * 4;
    if (!s_flag[r]) {  // no point in either row: skip the loads
      float2* d = W + r * S + y4;
      d[0] = d[1] = d[2] = d[3] = make_float2(0.f, 0.f);
      continue;
    }
    float4 a = *reinterpret_cast<const float4*>(g + (size_t)(2 * r) * N + y4);
    float4 b = *reinterpret_cast<const float4*>(g + (size_t)(2 * r + 1) * N + y4);
    if (cnt) {
      const float4 ca = *reinterpret_cast<const float4*>(cnt + (size_t)(2 * r) * N + y4);
      const float4 cb = *reinterpret_cast<const float4*>(cnt + (size_t)(2 * r + 1) * N + y4);
      a = make_float4(voxel_mean(a.x, ca.x), voxel_mean(a.y, ca.y), voxel_mean(a.z, ca.z), voxel_mean(a.w, ca.w));
      b = make_float4(voxel_mean(b.x, cb.x), voxel_mean(b.y, cb.y), voxel_mean(b.z, cb.z), voxel_mean(b.w, cb.w));
    }
    float2* d = W + r * S + y4;
    d[0] = make_float2(a.x, b.x);
    d[1] = make_float2(a.y, b.y);
    d[2] = make_float2(a.z, b.z);
    d[3] = make_float2(a.w, b.w);
    if ((a.x != 0.f) | (a.y != 0.f) | (a.z != 0.f) | (a.w != 0.f) | (b.x != 0.f) | (b.y != 0.f) | (b.z != 0.f) |
        (b.w != 0.f))
      s_live[r] = 1;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    int base = 0;
    for (int r0 = 0; r0 < NH; r0 += 32) {
      const bool live = r0 + (int)threadIdx.x < NH && s_live[r0 + threadIdx.x];
      const unsigned m = __ballot_sync(0xffffffffu, live);
      if (live) s_rows[base + __popc(m & ((1u << threadIdx.x) - 1u))] = r0 + threadIdx.x;
      base += __popc(m);
    }
    if (threadIdx.x == 0) s_nrows = base;
  }
  __syncthreads();
  const int nrows = s_nrows;
  float2* out = spec + (size_t)c * spec_cstride + (size_t)z * N * H2p;
  if (nrows == 0) {  // empty slab: its 2-D spectrum is zero
    for (int e = threadIdx.x; e < N * H2; e += T) {
      const int k = e / H2, ky = e - k * H2;
      out[(size_t)k * H2p + ky] = make_float2(0.f, 0.f);
    }
    if (nz && threadIdx.x == 0) *nz = 0;  // every thread read it before the barrier above
    return;
  }
  if (nz && threadIdx.x == 0) *nz = 1;
  // rows that are all zero stay zero under the y transform
  fft_tail<N, false, false, true, tail_threads<NF>()>(W, nrows, S, pN.tw, s_rows);  // over y, live rows
  fft_tail<NH, false, true, true, tail_threads<NF>()>(W, N, S, pH.tw);               // over r, columns
  for (int e = threadIdx.x; e < NH * H2; e += T) {
    const int k = e / H2, ky = e - k * H2;
    const float2 w1 = W[s_posH[k] * S + s_posN[ky]];
    const float2 w2 = W[s_posH[k == 0 ? 0 : NH - k] * S + s_posN[ky == 0 ? 0 : N - ky]];
    const float2 A = make_float2(0.5f * (w1.x + w2.x), 0.5f * (w1.y - w2.y));
    const float2 B = make_float2(0.5f * (w1.y + w2.y), -0.5f * (w1.x - w2.x));  // (w1 - conj w2) / 2i
    const float2 tB = cmul(__ldg(&pN.tw[k]), B);
    out[(size_t)k * H2p + ky] = cadd(A, tB);
    out[(size_t)(k + NH) * H2p + ky] = csub(A, tB);
  }
}

// Fused inverse of one z-slab: inverse over x and the real inverse over y of
// the product spectrum (natural kx), first-occurrence argmax of the signed
// output.  The ky = 0 and ky = N/2 columns are first projected onto their
// x-Hermitian parts, which is what a half-complex inverse reads (only the real
// parts of its DC and Nyquist terms after the inverse over x).
template <int NF>
__global__ void __launch_bounds__(tail_threads<NF>()) k_slab_inv(const float2* __restrict__ cspec, FftPlan pN,
                                                   FftPlan pH, unsigned long long* __restrict__ argmax,
                                                   float* __restrict__ volume, uint32_t limit) {
  constexpr int N = NF, NH = NF / 2, H2 = NF / 2 + 1, S = NF + 1;
  constexpr int T = tail_threads<NF>();  // the launch's block size
  const int H2p = spatial_h2p(N);
  extern __shared__ float2 W[];  // [NH][S]
  __shared__ int s_posN[N], s_posH[NH];  // digit-reversed positions of frequencies
  const int z = blockIdx.x;
  const float2* X = cspec + (size_t)z * N * H2p;
  for (int k = threadIdx.x; k < N; k += T) {
    s_posN[k] = fixed_freq2pos<N>(k);
    if (k < NH) s_posH[k] = fixed_freq2pos<NH>(k);
  }
  __syncthreads();
  // four elements' loads in flight per thread
  constexpr int U = 4;
  for (int e0 = threadIdx.x; e0 < NH * H2; e0 += U * T) {
    float2 x0u[U], x1u[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int e = e0 + u * T;
      const int k = e / H2, ky = e - k * H2;
      const bool ok = e < NH * H2;
      x0u[u] = ok ? X[(size_t)k * H2p + ky] : make_float2(0.f, 0.f);
      x1u[u] = ok ? X[(size_t)(k + NH) * H2p + ky] : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
    const int e = e0 + u * T;
    if (e >= NH * H2) break;
    const int k = e / H2, ky = e - k * H2;
    float2 x0 = x0u[u], x1 = x1u[u];
    if (ky == 0 || ky == NH) {
      const float2 m0 = X[(size_t)(k == 0 ? 0 : N - k) * H2p + ky];  // kx = -k
      const float2 m1 = X[(size_t)(NH - k) * H2p + ky];               // kx = -(k + N/2)
      x0 = make_float2(0.5f * (x0.x + m0.x), 0.5f * (x0.y - m0.y));
      x1 = make_float2(0.5f * (x1.x + m1.x), 0.5f * (x1.y - m1.y));
    }
    const float2 A = make_float2(0.5f * (x0.x + x1.x), 0.5f * (x0.y + x1.y));
    const float2 B = cmul(make_float2(0.5f * (x0.x - x1.x), 0.5f * (x0.y - x1.y)), cconj(__ldg(&pN.tw[k])));
    // W = A + i B at (k, ky); its mirror (-k, -ky) holds conj(A) + i conj(B)
    W[s_posH[k] * S + s_posN[ky]] = make_float2(A.x - B.y, A.y + B.x);
    if (ky >= 1 && ky < NH) W[s_posH[k == 0 ? 0 : NH - k] * S + s_posN[N - ky]] = make_float2(A.x + B.y, -A.y + B.x);
    }
  }
  __syncthreads();
  fft_tail<NH, true, true, true, tail_threads<NF>()>(W, N, S, pH.tw);    // over r, columns
  fft_tail<N, true, false, true, tail_threads<NF>()>(W, NH, S, pN.tw);   // over y, rows
  // per thread: the largest value, the lowest index among equal ones (the
  // reference's first occurrence, whatever order the thread visits them in)
  float bv = -INFINITY;
  uint32_t bi = 0xffffffffu;
  for (int e = threadIdx.x; e < NH * N; e += T) {
    const int r = e / N, y = e - r * N;
    const float2 v = W[r * S + y];
    const float a0 = 2.0f * v.x, a1 = 2.0f * v.y;
    const uint32_t i0 = (uint32_t)(((size_t)z * N + 2 * r) * N + y);
    const uint32_t i1 = i0 + N;
    if (i0 < limit && (a0 > bv || (a0 == bv && i0 < bi) || bi == 0xffffffffu)) {
      bv = a0;
      bi = i0;
    }
    if (i1 < limit && (a1 > bv || (a1 == bv && i1 < bi) || bi == 0xffffffffu)) {
      bv = a1;
      bi = i1;
    }
    if (volume) {
      volume[i0] = a0;
      volume[i1] = a1;
    }
  }
  warp_argmax_commit(bi == 0xffffffffu ? 0ull : pack_argmax(bv, bi), argmax);
}

// ---------------------------------------------------------------- launchers

constexpr int kMaxSmem = 227 * 1024;

// Opt-in dynamic shared memory: everything the static shared memory leaves.
static cudaError_t allow_max_smem(const void* fn) {
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, fn);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmem - (int)fa.sharedSizeBytes);
}

template <int NF>
static cudaError_t set_attrs() {
  cudaError_t e = allow_max_smem((const void*)k_fuse_z<NF>);
  if constexpr (NF > 0)
    if (e == cudaSuccess) e = allow_max_smem((const void*)k_fuse_z<NF, 6, 8>);
  if (e == cudaSuccess) e = allow_max_smem((const void*)k_r2c_y<NF>);
  if (e == cudaSuccess) e = allow_max_smem((const void*)k_fft_x<NF, false>);
  if (e == cudaSuccess) e = allow_max_smem((const void*)k_fft_x<NF, true>);
  if (e == cudaSuccess) e = allow_max_smem((const void*)k_c2r_y<NF>);
  return e;
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  return fn;
}

cudaError_t spatial_init_attributes() {
  cudaError_t e = cudaSuccess;
  for (int n : {64, 128, 200, 256, 320, 512, 0}) {  // every length PHGPU_DISPATCH_N instantiates
    cudaError_t r = cudaSuccess;
    PHGPU_DISPATCH_N(n, r = set_attrs<NF>());
    if (r != cudaSuccess) e = r;
  }
  for (auto fn : {(const void*)k_slab_fwd<64>, (const void*)k_slab_fwd<128>, (const void*)k_slab_fwd<200>,
                  (const void*)k_slab_inv<64>, (const void*)k_slab_inv<128>, (const void*)k_slab_inv<200>}) {
    cudaError_t r = allow_max_smem(fn);
    if (r != cudaSuccess) e = r;
  }
  // look the tensor-map encoder up now, not first inside a stream capture
  encode_tiled();
  return e;
}

bool spatial_slab_path(int N) { return N == 64 || N == 128 || N == 200; }

#define PHGPU_DISPATCH_SLAB(n, ...) \
  switch (n) {                      \
    case 64: {                      \
      constexpr int NF = 64;        \
      __VA_ARGS__;                  \
    } break;                        \
    case 128: {                     \
      constexpr int NF = 128;       \
      __VA_ARGS__;                  \
    } break;                        \
    default: {                      \
      constexpr int NF = 200;       \
      __VA_ARGS__;                  \
    } break;                        \
  }

// Tile width of the z pass: as many ky columns as fit (<= 8) in shared memory.
static size_t fuse_z_smem(int N, int A, int wt) {
  const int chunks = (N + 255) / 256;
  const size_t rows = (size_t)chunks * ((N + chunks - 1) / chunks);
  return rows * A * wt * sizeof(float2) + 16 + sizeof(FusionBands) + (size_t)N * sizeof(int);
}

bool fuse_z_tile_ok(int N, int A, int wt) {
  return (wt == 2 || wt == 4 || wt == 8 || wt == 16) && fuse_z_smem(N, A, wt) <= (size_t)kMaxSmem;
}

static int fuse_z_tile(int N, int A) {
  // >= 2: the loader moves two complex per 16-byte access, and a bulk copy's
  // innermost extent must be a multiple of 16 bytes
  int wt = 8;
  const int chunks = (N + 255) / 256;                       // bulk copies of <= 256 z rows
  const size_t rows = (size_t)chunks * ((N + chunks - 1) / chunks);
  const size_t extra = 16 + sizeof(FusionBands) + (size_t)N * sizeof(int);
  // narrower tiles until two blocks fit on an SM (one block cannot overlap
  // its bulk load with its own transforms), at least until the limit is met
  while (wt > 2 && rows * A * wt * sizeof(float2) + extra > (size_t)kMaxSmem / 2) wt >>= 1;
  return wt;
}

// cuTensorMapEncodeTiled through the runtime (no link against the driver
// library); null when unavailable, in which case the element loader is used.
cudaError_t launch_spatial_forward(const SpatialArgs& a, int side, cudaStream_t st) {
  const int N = a.N, H2 = N / 2 + 1;
  const size_t nv = (size_t)N * N * N;
  const size_t plane = (size_t)N * N * spatial_h2p(N);
  const float* grids = side == 0 ? a.grids_f : a.grids_g;
  const int nch = a.laplace ? a.n_data_ch : (a.lowpass ? 2 : 1);
  const float* count = a.grids_are_means ? nullptr : grids + (size_t)a.n_data_ch * nv;
  if (spatial_slab_path(N) && a.plan_half) {
    float2* spec = a.spec + (size_t)(side * a.n_data_ch) * plane;
    dim3 g(N, nch);
    const size_t sm = (size_t)(N / 2) * (N + 1) * sizeof(float2);
    const uint8_t* rowlive = side == 0 ? a.rowlive_f : a.rowlive_g;
    uint8_t* nz = a.slab_nz ? a.slab_nz + (size_t)(side * a.n_data_ch) * N : nullptr;
    PHGPU_DISPATCH_SLAB(N, k_slab_fwd<NF><<<g, tail_threads<NF>(), sm, st>>>(grids, nv, count, rowlive, spec, plane,
                                                                             *a.plan, *a.plan_half, nz));
    count_launches(1);
    return cudaGetLastError();
  }
  const int nrowblk = (int)((nv / N + kRowsR2C - 1) / kRowsR2C);
  for (int c = 0; c < nch; ++c) {
    float2* spec = a.spec + (size_t)(side * a.n_data_ch + c) * plane;
    const float* g = grids + (size_t)c * nv;
    dim3 gx((H2 + 15) / 16, N, 1);
    const uint8_t* rowlive = side == 0 ? a.rowlive_f : a.rowlive_g;
    const size_t smr = (size_t)(kRowsR2C / 2) * N * sizeof(float2) + (size_t)N * sizeof(int);
    PHGPU_DISPATCH_N(N,
        k_r2c_y<NF><<<nrowblk, 256, smr, st>>>(N, g, count, rowlive, spec, *a.plan);
        k_fft_x<NF, false><<<gx, 256, (size_t)N * 16 * sizeof(float2), st>>>(N, spec, *a.plan));
    count_launches(2);
  }
  return cudaGetLastError();
}

cudaError_t launch_spatial_fuse_z(const SpatialArgs& a, cudaStream_t st) {
  const int N = a.N, H2 = N / 2 + 1;
  const int A = a.laplace ? 2 * a.n_data_ch : 2;
  const int wt = fuse_z_tile_ok(N, A, a.fuse_tile) ? a.fuse_tile : fuse_z_tile(N, A);
  // bulk tensor copies of the [z][array][ky] tile (element = one complex)
  CUtensorMap tmap;
  memset(&tmap, 0, sizeof(tmap));
  FuseZTma tma{0, N, 1};
  if (EncodeTiledFn enc = encode_tiled()) {
    const size_t plane = (size_t)N * N * spatial_h2p(N);
    const int chunks = (N + 255) / 256;
    const int zbox = (N + chunks - 1) / chunks;
    const cuuint64_t dims[4] = {(cuuint64_t)spatial_h2p(N), (cuuint64_t)A, (cuuint64_t)N, (cuuint64_t)N};
    const cuuint64_t strides[3] = {(cuuint64_t)(a.laplace ? plane : plane * a.n_data_ch) * sizeof(float2),
                                   (cuuint64_t)spatial_h2p(N) * sizeof(float2),
                                   (cuuint64_t)N * spatial_h2p(N) * sizeof(float2)};
    const cuuint32_t box[4] = {(cuuint32_t)wt, (cuuint32_t)A, 1u, (cuuint32_t)zbox};
    const cuuint32_t estr[4] = {1u, 1u, 1u, 1u};
    void* base = (void*)(a.spec + (a.laplace ? 0 : (size_t)a.lowpass * plane));
    if (enc(&tmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, base, dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS)
      tma = FuseZTma{1, zbox, chunks};
  }
  const size_t rows = (size_t)tma.zbox * tma.chunks;
  const size_t smB = rows * A * wt * sizeof(float2) + 16 + sizeof(FusionBands) + (size_t)N * sizeof(int);
  if (smB > (size_t)kMaxSmem) return cudaErrorInvalidConfiguration;
  dim3 gB((H2 + wt - 1) / wt, N);
  const int xnat = (spatial_slab_path(N) && a.plan_half) ? 1 : 0;
  // the bench shape (Laplace fusion of three channels, tile width 8) has its
  // own instantiation with the tile shape known at compile time
  const bool shape68 = A == 6 && wt == 8;
  PHGPU_DISPATCH_N(N, {
    bool done = false;
    if constexpr (NF > 0) {
      if (shape68) {
        k_fuse_z<NF, 6, 8><<<gB, kFuseZThreads, smB, st>>>(a, *a.plan, wt, xnat, tmap, tma);
        done = true;
      }
    }
    if (!done) k_fuse_z<NF><<<gB, kFuseZThreads, smB, st>>>(a, *a.plan, wt, xnat, tmap, tma);
  });
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_spatial_inverse(const SpatialArgs& a, cudaStream_t st) {
  const int N = a.N, H2 = N / 2 + 1;
  const uint32_t limit = a.argmax_limit ? a.argmax_limit : 0xffffffffu;
  if (spatial_slab_path(N) && a.plan_half) {
    const size_t sm = (size_t)(N / 2) * (N + 1) * sizeof(float2);
    PHGPU_DISPATCH_SLAB(N, k_slab_inv<NF><<<N, tail_threads<NF>(), sm, st>>>(a.cspec, *a.plan, *a.plan_half, a.argmax,
                                                                             a.volume, limit));
    count_launches(1);
    return cudaGetLastError();
  }
  dim3 gC((H2 + 15) / 16, N, 1);
  const int nrowblk = (int)(((size_t)N * N + kRowsR2C - 1) / kRowsR2C);
  PHGPU_DISPATCH_N(N,
      k_fft_x<NF, true><<<gC, 256, (size_t)N * 16 * sizeof(float2), st>>>(N, a.cspec, *a.plan);
      k_c2r_y<NF><<<nrowblk, 256, (size_t)(kRowsR2C / 2) * N * sizeof(float2) + (size_t)N * sizeof(int), st>>>(
          N, a.cspec, *a.plan, a.argmax, a.volume, limit));
  count_launches(2);
  return cudaGetLastError();
}

cudaError_t launch_spatial_combine(const SpatialArgs& a, cudaStream_t st) {
  cudaError_t e = launch_spatial_fuse_z(a, st);
  if (e == cudaSuccess) e = launch_spatial_inverse(a, st);
  return e;
}

}  // namespace phgpu
