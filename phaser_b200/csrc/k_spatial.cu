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
#include "kernels.h"

namespace phgpu {

__device__ __forceinline__ int histc_bin(float x, const float* __restrict__ E, int N) {
  if (x < E[0] || x > E[N - 1]) return -1;
  int l = 0, h = N - 1, k = 0;
  while ((h - l) > 1) {
    k = (h + l) / 2;
    if (x < E[k])
      h = k;
    else
      l = k;
  }
  return (x == E[h]) ? h : l;
}

__global__ void k_voxelize(VoxelArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n_points) return;
  const float4 p = a.xyzi[i];
  float x = p.x, y = p.y, z = p.z;
  if (a.has_T) {
    // PCL 1.8 transformPointCloud order ((T0 x + T1 y) + T2 z) + T3
    const float* T = a.T;
    const float nx = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(T[0], x), __fmul_rn(T[1], y)), __fmul_rn(T[2], z)), T[3]);
    const float ny = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(T[4], x), __fmul_rn(T[5], y)), __fmul_rn(T[6], z)), T[7]);
    const float nz = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(T[8], x), __fmul_rn(T[9], y)), __fmul_rn(T[10], z)), T[11]);
    x = nx;
    y = ny;
    z = nz;
  }
  const uint32_t N = (uint32_t)a.N;
  const uint32_t bx = (uint32_t)histc_bin(x, a.edges, a.N);
  const uint32_t by = (uint32_t)histc_bin(y, a.edges, a.N);
  const uint32_t bz = (uint32_t)histc_bin(z, a.edges, a.N);
  const uint32_t lin = (bx * N + by) + (N * N * bz);
  const uint32_t nv = N * N * N;
  const bool ok = lin < nv;
  if (a.lin_out) a.lin_out[i] = ok ? lin : 0xffffffffu;
  if (!ok) return;
  float* g = a.grids;
  atomicAdd(&g[lin], p.w);
  const float r = sqrtf(__fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z)));
  atomicAdd(&g[(size_t)nv + lin], r);
  if (a.n_data_ch > 2) atomicAdd(&g[(size_t)2 * nv + lin], a.refl ? a.refl[i] : 0.0f);
  if (a.n_data_ch > 3) atomicAdd(&g[(size_t)3 * nv + lin], a.amb ? a.amb[i] : 0.0f);
  atomicAdd(&g[(size_t)a.n_data_ch * nv + lin], 1.0f);
}

cudaError_t launch_voxelize(const VoxelArgs& a, cudaStream_t st) {
  if (a.n_points > 0) k_voxelize<<<(a.n_points + 255) / 256, 256, 0, st>>>(a);
  return cudaGetLastError();
}

// ---------------------------------------------------------------- A1
// rows r = z*N + x of one channel; out spec[ch][r][ky], ky in [0, N/2].
__global__ void k_r2c_y(int N, const float* __restrict__ grid, const float* __restrict__ count,
                        float2* __restrict__ spec, FftPlan plan) {
  extern __shared__ float2 rows[];
  constexpr int R = 8;
  const int H2 = N / 2 + 1;
  const size_t nrows = (size_t)N * N;
  const size_t r0 = (size_t)blockIdx.x * R;
  for (int e = threadIdx.x; e < R * N; e += blockDim.x) {
    const int rr = e / N, y = e % N;
    const size_t r = r0 + rr;
    float v = 0.0f;
    if (r < nrows) {
      v = grid[r * N + y];
      if (count) {
        const float q = v / count[r * N + y];
        v = isfinite(q) ? q : 0.0f;
      }
    }
    rows[e] = make_float2(v, 0.0f);
  }
  __syncthreads();
  fft_smem<false>(rows, R, N, 1, plan);
  for (int e = threadIdx.x; e < R * H2; e += blockDim.x) {
    const int rr = e / H2, ky = e % H2;
    const size_t r = r0 + rr;
    if (r < nrows) spec[r * H2 + ky] = rows[rr * N + fft_freq2pos(ky, plan)];
  }
}

// ---------------------------------------------------------------- A2 / C1
// In-place transform along x for a tile of ky at one z: spec[z][x][ky].
template <bool INV>
__global__ void k_fft_x(int N, float2* __restrict__ spec, FftPlan plan) {
  extern __shared__ float2 tile[];
  constexpr int Wt = 16;
  const int H2 = N / 2 + 1;
  const int ky0 = blockIdx.x * Wt;
  const int wt = min(Wt, H2 - ky0);
  float2* base = spec + (size_t)blockIdx.z * N * N * H2 + (size_t)blockIdx.y * N * H2;
  for (int e = threadIdx.x; e < N * Wt; e += blockDim.x) {
    const int x = e / Wt, t = e % Wt;
    tile[e] = t < wt ? base[(size_t)x * H2 + ky0 + t] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  fft_smem<INV>(tile, Wt, 1, Wt, plan);
  for (int e = threadIdx.x; e < N * Wt; e += blockDim.x) {
    const int x = e / Wt, t = e % Wt;
    if (t < wt) base[(size_t)x * H2 + ky0 + t] = tile[e];
  }
}

// ---------------------------------------------------------------- B
// For one x position (digit-reversed) and a tile of ky: forward z FFT of all
// 2C arrays, fusion + cross power, inverse z FFT of the product.
__global__ void k_fuse_z(SpatialArgs a, FftPlan plan, int Wt) {
  extern __shared__ float2 tile[];  // [z][arr][t]
  const int N = a.N, H2 = N / 2 + 1;
  const int C = a.n_data_ch;
  const int A = a.laplace ? 2 * C : 2;
  const int ky0 = blockIdx.x * Wt;
  const int wt = min(Wt, H2 - ky0);
  const int xp = blockIdx.y;
  const size_t plane = (size_t)N * N * H2;
  const int rowlen = A * Wt;
  for (int e = threadIdx.x; e < N * rowlen; e += blockDim.x) {
    const int z = e / rowlen, rem = e % rowlen, ar = rem / Wt, t = rem % Wt;
    // arrays: f channels 0..C-1 then g channels; plain mode uses channel 0 of each side
    const int src = a.laplace ? ar : (ar == 0 ? 0 : C);
    tile[e] = t < wt ? a.spec[(size_t)src * plane + ((size_t)z * N + xp) * H2 + ky0 + t]
                     : make_float2(0.f, 0.f);
  }
  __syncthreads();
  fft_smem<false>(tile, rowlen, 1, rowlen, plan);
  const int kx = fft_pos2freq(xp, plan);
  const uint32_t nv = (uint32_t)N * (uint32_t)N * (uint32_t)N;
  for (int e = threadIdx.x; e < N * Wt; e += blockDim.x) {
    const int zp = e / Wt, t = e % Wt;
    float2* row = tile + (size_t)zp * rowlen;
    float2 F, G;
    if (!a.laplace) {
      F = row[t];
      G = row[Wt + t];
    } else {
      const int kz = fft_pos2freq(zp, plan);
      const uint32_t klin = ((uint32_t)kz * N + (uint32_t)kx) * (uint32_t)H2 + (uint32_t)(ky0 + t);
      const uint32_t p = (uint32_t)(((uint64_t)klin + (nv >> 1)) % nv);
      const int op = fusion_op(p, a.bands);
      if (op == kFuseZero) {
        F = make_float2(0.f, 0.f);
        G = F;
      } else if (op == kFuseMean) {
        float fr = 0.f, fi = 0.f, gr = 0.f, gi = 0.f;
        for (int c = 0; c < C; ++c) {
          fr += row[c * Wt + t].x;
          fi += row[c * Wt + t].y;
          gr += row[(C + c) * Wt + t].x;
          gi += row[(C + c) * Wt + t].y;
        }
        const float inv = (float)a.n_total_ch;
        F = make_float2(fr / inv, fi / inv);
        G = make_float2(gr / inv, gi / inv);
      } else {
        float bf = -1.f, bg = -1.f;
        F = G = make_float2(0.f, 0.f);
        for (int c = 0; c < C; ++c) {
          const float2 u = row[c * Wt + t];
          const float2 v = row[(C + c) * Wt + t];
          const float eu = u.x * u.x + u.y * u.y;
          const float ev = v.x * v.x + v.y * v.y;
          if (eu > bf) {
            bf = eu;
            F = u;
          }
          if (ev > bg) {
            bg = ev;
            G = v;
          }
        }
      }
    }
    // complexMulSeq: C = F * conj(G)
    const float2 prod = make_float2(F.x * G.x - F.y * (-G.y), F.x * (-G.y) + F.y * G.x);
    row[t] = prod;  // only this thread reads or writes position (zp, t)
  }
  __syncthreads();
  fft_smem<true>(tile, Wt, 1, rowlen, plan);
  for (int e = threadIdx.x; e < N * Wt; e += blockDim.x) {
    const int z = e / Wt, t = e % Wt;
    if (t < wt) a.cspec[((size_t)z * N + xp) * H2 + ky0 + t] = tile[(size_t)z * rowlen + t];
  }
}

// ---------------------------------------------------------------- C2
__global__ void k_c2r_y(int N, const float2* __restrict__ cspec, FftPlan plan,
                        unsigned long long* __restrict__ argmax, float* __restrict__ volume) {
  extern __shared__ float2 rows[];
  constexpr int R = 8;
  const int H2 = N / 2 + 1;
  const size_t nrows = (size_t)N * N;
  const size_t r0 = (size_t)blockIdx.x * R;
  for (int e = threadIdx.x; e < R * N; e += blockDim.x) rows[e] = make_float2(0.f, 0.f);
  __syncthreads();
  const int hmax = (N - 1) / 2;  // last ky with a mirrored partner
  for (int e = threadIdx.x; e < R * H2; e += blockDim.x) {
    const int rr = e / H2, ky = e % H2;
    const size_t r = r0 + rr;
    if (r >= nrows) continue;
    const float2 v = cspec[r * H2 + ky];
    float2* row = rows + rr * N;
    row[fft_freq2pos(ky, plan)] = v;
    if (ky >= 1 && ky <= hmax) row[fft_freq2pos(N - ky, plan)] = cconj(v);
  }
  __syncthreads();
  fft_smem<true>(rows, R, N, 1, plan);
  unsigned long long best = 0ull;
  for (int e = threadIdx.x; e < R * N; e += blockDim.x) {
    const int rr = e / N, y = e % N;
    const size_t r = r0 + rr;
    if (r < nrows) {
      const float v = rows[e].x;
      const uint32_t idx = (uint32_t)(r * N + y);
      const unsigned long long key = pack_argmax(v, idx);
      best = key > best ? key : best;
      if (volume) volume[idx] = v;
    }
  }
  warp_argmax_commit(best, argmax);
}

// ---------------------------------------------------------------- launchers

constexpr int kMaxSmem = 227 * 1024;

cudaError_t spatial_init_attributes() {
  cudaError_t e = cudaFuncSetAttribute(k_fuse_z, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmem);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_r2c_y, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmem);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fft_x<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmem);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fft_x<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmem);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_c2r_y, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmem);
  return e;
}

// Tile width of the z pass: as many ky columns as fit (<= 8) in shared memory.
static int fuse_z_tile(int N, int A) {
  int wt = 8;
  while (wt > 1 && (size_t)N * A * wt * sizeof(float2) > (size_t)kMaxSmem) wt >>= 1;
  return wt;
}

cudaError_t launch_spatial_forward(const SpatialArgs& a, int side, cudaStream_t st) {
  const int N = a.N, H2 = N / 2 + 1;
  const size_t nv = (size_t)N * N * N;
  const size_t plane = (size_t)N * N * H2;
  const float* grids = side == 0 ? a.grids_f : a.grids_g;
  const int nch = a.laplace ? a.n_data_ch : 1;
  const float* count = a.grids_are_means ? nullptr : grids + (size_t)a.n_data_ch * nv;
  const int nrowblk = (int)((nv / N + 7) / 8);
  for (int c = 0; c < nch; ++c) {
    float2* spec = a.spec + (size_t)(side * a.n_data_ch + c) * plane;
    k_r2c_y<<<nrowblk, 256, (size_t)8 * N * sizeof(float2), st>>>(N, grids + (size_t)c * nv, count, spec, *a.plan);
    dim3 g((H2 + 15) / 16, N, 1);
    k_fft_x<false><<<g, 256, (size_t)N * 16 * sizeof(float2), st>>>(N, spec, *a.plan);
  }
  return cudaGetLastError();
}

cudaError_t launch_spatial_combine(const SpatialArgs& a, cudaStream_t st) {
  const int N = a.N, H2 = N / 2 + 1;
  const int A = a.laplace ? 2 * a.n_data_ch : 2;
  const int wt = fuse_z_tile(N, A);
  const size_t smB = (size_t)N * A * wt * sizeof(float2);
  if (smB > (size_t)kMaxSmem) return cudaErrorInvalidConfiguration;
  dim3 gB((H2 + wt - 1) / wt, N);
  k_fuse_z<<<gB, 256, smB, st>>>(a, *a.plan, wt);
  dim3 gC((H2 + 15) / 16, N, 1);
  k_fft_x<true><<<gC, 256, (size_t)N * 16 * sizeof(float2), st>>>(N, a.cspec, *a.plan);
  const int nrowblk = (int)(((size_t)N * N + 7) / 8);
  k_c2r_y<<<nrowblk, 256, (size_t)8 * N * sizeof(float2), st>>>(N, a.cspec, *a.plan, a.argmax, a.volume);
  return cudaGetLastError();
}

}  // namespace phgpu
