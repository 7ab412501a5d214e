// S^2 sampling on the GPU: spherical projection of each point and exact 1-NN
// of every Driscoll-Healy grid direction among the projected points.
//
// Reference behaviour: SphericalProjection::naiveProjection
// (phaser_common/src/common/spherical-projection.cc:19-41) and
// PointCloud::getNearestPoints / sampleNearestWithoutCloudInfo
// (phaser_common/src/model/point-cloud.cc:93-157).  Distances are float L2^2
// accumulated as ((dx^2 + dy^2) + dz^2) without contraction; the lowest point
// index wins exact ties; a match farther than the squared voxel size is
// dropped (all channels 0).
//
// Search structure: the projected points are counting-sorted by the grid's
// own (theta, phi) bins -- row i covers colatitudes [i, i + 1) pi / 2B,
// column j longitudes within pi / 2B of 2 pi j / 2B -- so every bin, and
// every run of neighbouring columns of a row, is one contiguous point range.
// A direction (i, j), one group of 8 lanes, sweeps the non-empty rows outward from its
// own row while the row's colatitude distance |theta_q - row| can still beat
// the bound; the first row reached is probed at columns j-1..j+1 for a
// finite bound, and in each row only the columns whose longitudes lie within
// the bound's spherical cap are scanned (the cap's longitude half-width at
// the row's colatitudes).  A LiDAR scan needs about two rows and fifty
// points per direction, so the search is a short chain of dependent loads
// per direction, run for all directions at once.  The bound is kept as an
// upper bound hb of hav(beta) = sin^2(beta / 2) of the best distance's angle
// inflated by 1e-4 rad, and a row's window follows from the haversine law
//   hav(d) = hav(t - t_q) + sin t sin t_q hav(dphi)
// with per-row tables (sin of the row edges, hav of the row's colatitude
// distance) deflated by margins far above the float rounding of the unit
// vectors, so no point that could be (or tie) the nearest is ever skipped:
// the search is exact whatever bound it starts from.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "kernels.h"

namespace phgpu {

// float functions evaluated in double and rounded once (correctly rounded
// except in rare near-halfway cases; glibc's float versions can differ by one
// ulp, so projected coordinates match the reference with high probability).
__device__ __forceinline__ float acos_f(float x) { return (float)acos((double)x); }
__device__ __forceinline__ float atan2_f(float y, float x) { return (float)atan2((double)y, (double)x); }

// Projection of every point, its bin and the per-bin and per-row counts.
__global__ void k_project(const float4* __restrict__ xyzi, int P, float4* __restrict__ proj,
                          double* __restrict__ range, uint32_t* __restrict__ key, int n2b,
                          uint32_t* __restrict__ bin_count, uint32_t* __restrict__ row_count,
                          const uint32_t* __restrict__ P_dev) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (P_dev ? (int)*P_dev : P)) return;
  const float4 p = xyzi[i];
  const float sxy = __fadd_rn(__fmul_rn(p.x, p.x), __fmul_rn(p.y, p.y));
  const double dist_xy = (double)sqrtf(sxy);
  const float zz = __fmul_rn(p.z, p.z);
  const double dist = sqrt(__dadd_rn(__dmul_rn(dist_xy, dist_xy), (double)zz));
  const float oz = (float)__ddiv_rn((double)p.z, dist);
  const double tx = (double)acos_f(oz);
  const double ty = fmod(__dadd_rn((double)atan2_f(p.y, p.x), 2.0 * M_PI), 2.0 * M_PI);
  double st, ct, sp, cp;
  sincos(tx, &st, &ct);
  sincos(ty, &sp, &cp);
  const float ox = (float)__dmul_rn(st, cp);
  const float oy = (float)__dmul_rn(st, sp);
  proj[i] = make_float4(ox, oy, oz, 0.0f);
  range[i] = dist;
  // points at the origin or with non-finite coordinates have no direction:
  // they are left out of the search structure
  if (!(isfinite(ox) && isfinite(oy) && isfinite(oz))) {
    key[i] = 0xffffffffu;
    return;
  }
  const double w = M_PI / (double)n2b;  // bin height in theta, half bin width in phi
  const int bi = min(max((int)(tx / w), 0), n2b - 1);
  int bj = (int)floor(ty / (2.0 * w) + 0.5);
  bj = bj >= n2b ? bj - n2b : max(bj, 0);
  const uint32_t b = (uint32_t)(bi * n2b + bj);
  key[i] = b;
  // consecutive points of a scan mostly share bins and rows: one atomic per
  // group of lanes with the same key
  {
    const unsigned act = __activemask();
    const int lane = threadIdx.x & 31;
    const unsigned pb = __match_any_sync(act, b);
    if (lane == __ffs(pb) - 1) atomicAdd(&bin_count[b], (uint32_t)__popc(pb));
    const unsigned pr = __match_any_sync(act, bi);
    if (lane == __ffs(pr) - 1) atomicAdd(&row_count[bi], (uint32_t)__popc(pr));
  }
}

// Bin starts and row tables.  Block r: the exclusive scan of row r's n2b bin
// counts offset by the points of rows < r; row_nxt[r] = first non-empty row
// >= r (n2b if none), row_prv[r] = last non-empty row < r (-1 if none).
constexpr int kBinScanThreads = 256;
constexpr int kMaxGridSide = 1024;  // 2B for B <= 512

// Also the row tables of the window bound: sin_tab[r] = sin(r w) - 1e-5
// (clamped at 0) for the row edges r = 0..2B, hav_tab[d] = hav((d - 1/2) w)
// (1 - 1e-4) for the colatitude distance of a row d >= 1 rows away
// (hav_tab[0] = 0), w = pi / 2B.
__global__ void __launch_bounds__(kBinScanThreads) k_bin_scan(int n2b, const uint32_t* __restrict__ bin_count,
                                                              const uint32_t* __restrict__ row_count,
                                                              uint32_t* __restrict__ bin_start,
                                                              int* __restrict__ row_nxt, int* __restrict__ row_prv,
                                                              float* __restrict__ sin_tab, float* __restrict__ hav_tab) {
  __shared__ uint32_t s_rows[kMaxGridSide];
  __shared__ uint32_t s_w[kBinScanThreads / 32];
  __shared__ uint32_t s_base;
  const int r = blockIdx.x, t = threadIdx.x, lane = t & 31, warp = t >> 5;
  uint32_t part = 0;
  for (int q = t; q < n2b; q += kBinScanThreads) {
    const uint32_t v = __ldg(&row_count[q]);
    s_rows[q] = v;
    part += q < r ? v : 0u;
  }
  for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
  if (lane == 0) s_w[warp] = part;
  __syncthreads();
  if (t == 32) {
    const double w = M_PI / (double)n2b;
    sin_tab[r] = fmaxf((float)sin(r * w) - 1e-5f, 0.0f);
    if (r == n2b - 1) sin_tab[n2b] = 0.0f;
    const double h = sin(0.5 * (r - 0.5) * w);
    hav_tab[r] = r == 0 ? 0.0f : (float)(h * h) * (1.0f - 1e-4f);
  }
  if (t == 0) {
    uint32_t b = 0;
    for (int k = 0; k < kBinScanThreads / 32; ++k) b += s_w[k];
    s_base = b;
    int nx = r;
    while (nx < n2b && s_rows[nx] == 0u) ++nx;
    row_nxt[r] = nx;
    int pv = r - 1;
    while (pv >= 0 && s_rows[pv] == 0u) --pv;
    row_prv[r] = pv;
    if (r == n2b - 1) {
      row_nxt[n2b] = n2b;
      row_prv[n2b] = s_rows[r] ? r : pv;
    }
  }
  __syncthreads();
  // row scan: thread t owns columns [t * per, (t + 1) * per)
  const int per = (n2b + kBinScanThreads - 1) / kBinScanThreads;
  const uint32_t* rc = bin_count + (size_t)r * n2b;
  const int c_lo = min(n2b, t * per), c_hi = min(n2b, (t + 1) * per);
  uint32_t sum = 0;
  for (int c = c_lo; c < c_hi; ++c) sum += __ldg(&rc[c]);
  uint32_t incl = sum;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  __syncthreads();
  if (lane == 31) s_w[warp] = incl;
  __syncthreads();
  uint32_t run = s_base + incl - sum;
  for (int k = 0; k < warp; ++k) run += s_w[k];
  uint32_t* bs = bin_start + (size_t)r * n2b;
  for (int c = c_lo; c < c_hi; ++c) {
    bs[c] = run;
    run += __ldg(&rc[c]);
  }
  if (r == n2b - 1 && t == kBinScanThreads - 1) bin_start[(size_t)n2b * n2b] = run;
}

// Counting-sort scatter: sorted[k] = {x, y, z, point index (bits)}.
__global__ void k_bin_scatter(int P, const float4* __restrict__ proj, const uint32_t* __restrict__ key,
                              const uint32_t* __restrict__ bin_start, uint32_t* __restrict__ cursor,
                              float4* __restrict__ sorted, const uint32_t* __restrict__ P_dev) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (P_dev ? (int)*P_dev : P)) return;
  const uint32_t k = key[i];
  if (k == 0xffffffffu) return;
  const unsigned act = __activemask();
  const int lane = threadIdx.x & 31;
  const unsigned peers = __match_any_sync(act, k);
  const int leader = __ffs(peers) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(&cursor[k], (uint32_t)__popc(peers));
  base = __shfl_sync(peers, base, leader);
  const uint32_t slot = bin_start[k] + base + __popc(peers & ((1u << lane) - 1u));
  const float4 p = proj[i];
  sorted[slot] = make_float4(p.x, p.y, p.z, __int_as_float(i));
}

__device__ __forceinline__ float ref_dist2(float qx, float qy, float qz, float4 p) {
  const float dx = __fsub_rn(qx, p.x);
  const float dy = __fsub_rn(qy, p.y);
  const float dz = __fsub_rn(qz, p.z);
  float r = __fmul_rn(dx, dx);
  r = __fadd_rn(r, __fmul_rn(dy, dy));
  r = __fadd_rn(r, __fmul_rn(dz, dz));
  return r;
}

__device__ __forceinline__ void nn_update(float d, int idx, float& best, int& bidx) {
  if (d < best || (d == best && idx < bidx)) {
    best = d;
    bidx = idx;
  }
}

// Writes the sampled channels {range, intensity, reflectivity, ambient}
// (float) of the nearest point into out[ch][qi] for ch < n_out_ch and its
// index (or -1) into nn_idx; a match farther than max_sq is dropped.
__device__ __forceinline__ void emit_sample(int qi, int nq, float best, int bidx, float max_sq,
                                            const float4* __restrict__ xyzi, const double* __restrict__ range,
                                            const float* __restrict__ refl, const float* __restrict__ amb,
                                            int n_out_ch, float* __restrict__ out, int32_t* __restrict__ nn_idx) {
  const bool ok = (bidx != 0x7fffffff) && !(best > max_sq);
  float v[4] = {0.f, 0.f, 0.f, 0.f};
  if (ok) {
    v[0] = (float)range[bidx];
    v[1] = xyzi[bidx].w;
    v[2] = refl ? refl[bidx] : 0.0f;
    v[3] = amb ? amb[bidx] : 0.0f;
  }
  for (int c = 0; c < n_out_ch; ++c) out[(size_t)c * nq + qi] = v[c];
  if (nn_idx) nn_idx[qi] = ok ? bidx : -1;
}


// ---------------------------------------------------------------- row sweep
constexpr float kAngleMargin = 1e-4f;

// Upper bound of sin^2(beta / 2) for the angle beta of a float squared chord
// inflated by kAngleMargin (sin(asin h + m / 2) <= h + m / 2), so float
// rounding of the unit vectors cannot hide a nearer point; 2 (> 1) when the
// chord bounds nothing.
__device__ __forceinline__ float hav_of_l2(float best) {
  if (!(best < 3.99f)) return 2.0f;
  const float s = 0.5f * sqrtf(best) * (1.0f + kAngleMargin) + 0.5f * kAngleMargin;
  return s >= 1.0f ? 2.0f : s * s;
}

// Lanes per direction: a group of kGroup lanes strides over the points of a
// window (coalesced 16-byte loads), then reduces its minima.
constexpr int kGroup = 8;

// Scans columns c0 .. c0 + len - 1 (mod n2b) of row r: lane g of the group
// takes points g, g + kGroup, ... (two in flight); lane-private minima.
__device__ __forceinline__ void scan_cols(int r, int c0, int len, int n2b, int g, float qx, float qy, float qz,
                                          const uint32_t* __restrict__ bin_start, const float4* __restrict__ sorted,
                                          float& best, int& bidx) {
  if (len <= 0) return;
  c0 = c0 < 0 ? c0 + n2b : (c0 >= n2b ? c0 - n2b : c0);
  const uint32_t* rs = bin_start + (size_t)r * n2b;
  const int e0 = min(c0 + len, n2b);
  uint32_t seg[4] = {__ldg(&rs[c0]), __ldg(&rs[e0]), 0u, 0u};
  if (c0 + len > n2b) {
    seg[2] = __ldg(&rs[0]);
    seg[3] = __ldg(&rs[c0 + len - n2b]);
  }
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const uint32_t e = seg[2 * h + 1];
    uint32_t k = seg[2 * h] + g;
    for (; k + kGroup < e; k += 2 * kGroup) {
      const float4 p0 = __ldg(&sorted[k]), p1 = __ldg(&sorted[k + kGroup]);
      nn_update(ref_dist2(qx, qy, qz, p0), __float_as_int(p0.w), best, bidx);
      nn_update(ref_dist2(qx, qy, qz, p1), __float_as_int(p1.w), best, bidx);
    }
    if (k < e) {
      const float4 p0 = __ldg(&sorted[k]);
      nn_update(ref_dist2(qx, qy, qz, p0), __float_as_int(p0.w), best, bidx);
    }
  }
}

// Minimum (distance, then index) over the group; every lane gets it.
__device__ __forceinline__ void group_nn_min(unsigned gmask, float& best, int& bidx) {
#pragma unroll
  for (int o = kGroup / 2; o > 0; o >>= 1) {
    const float ob = __shfl_xor_sync(gmask, best, o);
    const int oi = __shfl_xor_sync(gmask, bidx, o);
    nn_update(ob, oi, best, bidx);
  }
}

// Half-width k (in columns) of the cap window of row r, d rows from the
// direction's own row: column j +- c holds longitudes at least (c - 1/2) 2w
// away from phi_q, and a point of the row within the bound has
//   hav(dphi) <= (hb - hav(row distance)) / (min(sin a, sin b) sin t_q)
// (sin is concave, so its minimum over the row's colatitudes [a, b] is at an
// edge).  n2b: the whole row.
__device__ __forceinline__ int row_window(int r, int d, int n2b, float w, float stq, float hb,
                                          const float* __restrict__ sin_tab, const float* __restrict__ hav_tab) {
  if (hb >= 1.0f) return n2b;
  const float num = hb - __ldg(&hav_tab[d]);
  const float den = fminf(__ldg(&sin_tab[r]), __ldg(&sin_tab[r + 1])) * stq;
  if (!(num < den)) return n2b;  // the bound reaches every longitude (or a pole row)
  if (num <= 0.0f) return 0;
  const float e = 2.0f * asinf(sqrtf(num / den)) + kAngleMargin;
  const float kf = e / (2.0f * w) + 0.5f;
  return kf >= (float)n2b ? n2b : (int)kf;
}

constexpr int kQueryThreads = 256;

// One group of kGroup lanes per direction of the 2B x 2B grid: the
// non-empty rows are visited outward from the direction's own row, nearest
// colatitude first, while their colatitude distance can beat the bound.  The
// first row visited is probed at columns j - 1 .. j + 1 to make the bound
// finite; every row's columns within the bound's cap are then scanned (the
// probed ones once).  Control flow is uniform within a group.  Six blocks per
// SM (40 registers, no spills) hide more of the dependent-load latency than
// the four that 64 registers allowed (s2_sample 0.0484 vs 0.0510 ms per cloud
// at B = 100).
__global__ void __launch_bounds__(kQueryThreads, 6)
k_nn_rows(int n2b, const float4* __restrict__ grid, const float4* __restrict__ sorted,
          const uint32_t* __restrict__ bin_start, const int* __restrict__ row_nxt, const int* __restrict__ row_prv,
          const float* __restrict__ sin_tab, const float* __restrict__ hav_tab, float max_sq,
          const float4* __restrict__ xyzi, const double* __restrict__ range, const float* __restrict__ refl,
          const float* __restrict__ amb, int n_out_ch, float* __restrict__ out, int32_t* __restrict__ nn_idx) {
  const int nq = n2b * n2b;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int qi = tid / kGroup, g = tid % kGroup;
  if (qi >= nq) return;  // whole groups: nq * kGroup threads are launched in full groups
  const unsigned gmask = ((1u << kGroup) - 1u) << ((threadIdx.x & 31) & ~(kGroup - 1));
  const float w = 3.14159265358979f / (float)n2b;
  const float4 q = __ldg(&grid[qi]);
  const int i = qi / n2b, j = qi - i * n2b;
  // sin t_q of the direction's colatitude (i + 1/2) w, deflated like the table
  const float stq = fmaxf(sinf(((float)i + 0.5f) * w) - 1e-5f, 0.0f);
  float best = INFINITY;
  int bidx = 0x7fffffff;
  float hb = 2.0f;
  int up = __ldg(&row_nxt[i]), dn = __ldg(&row_prv[i]);
  bool probed = false;
  for (;;) {
    if (up >= n2b && dn < 0) break;
    const int du = up < n2b ? up - i : 0x7fffffff, dd = dn >= 0 ? i - dn : 0x7fffffff;
    const bool take_up = du <= dd;
    const int d = take_up ? du : dd;
    // the row's colatitude distance alone must not exceed the bound
    if (!(__ldg(&hav_tab[d]) <= hb)) break;
    const int r = take_up ? up : dn;
    if (!probed) {
      const int pw = min(3, n2b);
      scan_cols(r, j - 1, pw, n2b, g, q.x, q.y, q.z, bin_start, sorted, best, bidx);
      group_nn_min(gmask, best, bidx);
      hb = hav_of_l2(best);
      const int k = row_window(r, d, n2b, w, stq, hb, sin_tab, hav_tab);
      if (2 * k + 1 >= n2b) {
        scan_cols(r, j + 2, n2b - pw, n2b, g, q.x, q.y, q.z, bin_start, sorted, best, bidx);
      } else if (k >= 2) {
        scan_cols(r, j - k, k - 1, n2b, g, q.x, q.y, q.z, bin_start, sorted, best, bidx);
        scan_cols(r, j + 2, k - 1, n2b, g, q.x, q.y, q.z, bin_start, sorted, best, bidx);
      }
      probed = true;
    } else {
      const int k = row_window(r, d, n2b, w, stq, hb, sin_tab, hav_tab);
      if (2 * k + 1 >= n2b)
        scan_cols(r, 0, n2b, n2b, g, q.x, q.y, q.z, bin_start, sorted, best, bidx);
      else
        scan_cols(r, j - k, 2 * k + 1, n2b, g, q.x, q.y, q.z, bin_start, sorted, best, bidx);
    }
    group_nn_min(gmask, best, bidx);
    hb = hav_of_l2(best);
    if (take_up)
      up = __ldg(&row_nxt[up + 1]);
    else
      dn = __ldg(&row_prv[dn]);
  }
  if (g == 0) emit_sample(qi, nq, best, bidx, max_sq, xyzi, range, refl, amb, n_out_ch, out, nn_idx);
}

// ---------------------------------------------------------------- launcher

std::atomic<unsigned long long> g_launch_count{0};
thread_local int g_capture_depth = 0;

namespace {
int grid_side(int max_queries) {
  int n = (int)sqrt((double)max_queries);
  while ((long long)n * n < max_queries) ++n;
  return n;
}
}  // namespace

size_t sampler_scratch_bytes(int max_points, int max_queries) {
  const int n2b = grid_side(max_queries);
  const size_t nbins = (size_t)n2b * n2b;
  size_t b = (size_t)max_points * sizeof(float4);                // proj
  b += (size_t)max_points * sizeof(double);                      // range
  b += (size_t)max_points * sizeof(uint32_t);                    // key
  b += (size_t)max_points * sizeof(float4);                      // sorted
  b += (2 * nbins + (size_t)n2b) * sizeof(uint32_t);             // bin counts, cursors, row counts
  b += (nbins + 1) * sizeof(uint32_t);                           // bin starts
  b += 2 * (size_t)(n2b + 1) * sizeof(int);                      // row tables
  b += 2 * (size_t)(n2b + 1) * sizeof(float);                    // window bound tables
  return b + 10 * 256;  // carve() rounds each region up to 256 bytes
}

static inline char* carve(char*& p, size_t bytes) {
  char* r = p;
  p += (bytes + 255) & ~(size_t)255;
  return r;
}

cudaError_t launch_sample(const SampleArgs& a, cudaStream_t st) {
  const int n2b = a.n2b;
  if (n2b <= 0 || n2b > kMaxGridSide || (size_t)n2b * n2b != (size_t)a.n_queries) return cudaErrorInvalidValue;
  const size_t nbins = (size_t)n2b * n2b;
  char* p = (char*)a.scratch;
  float4* proj = (float4*)carve(p, (size_t)a.max_points * sizeof(float4));
  double* range = (double*)carve(p, (size_t)a.max_points * sizeof(double));
  uint32_t* key = (uint32_t*)carve(p, (size_t)a.max_points * sizeof(uint32_t));
  float4* sorted = (float4*)carve(p, (size_t)a.max_points * sizeof(float4));
  uint32_t* counts = (uint32_t*)carve(p, (2 * nbins + (size_t)n2b) * sizeof(uint32_t));
  uint32_t* bin_count = counts;
  uint32_t* cursor = counts + nbins;
  uint32_t* row_count = counts + 2 * nbins;
  uint32_t* bin_start = (uint32_t*)carve(p, (nbins + 1) * sizeof(uint32_t));
  int* row_nxt = (int*)carve(p, (size_t)(n2b + 1) * sizeof(int));
  int* row_prv = (int*)carve(p, (size_t)(n2b + 1) * sizeof(int));
  float* sin_tab = (float*)carve(p, (size_t)(n2b + 1) * sizeof(float));
  float* hav_tab = (float*)carve(p, (size_t)(n2b + 1) * sizeof(float));

  cudaMemsetAsync(counts, 0, (2 * nbins + (size_t)n2b) * sizeof(uint32_t), st);
  const int P = a.n_points;
  int launched = 0;
  if (P > 0) {
    k_project<<<(P + 255) / 256, 256, 0, st>>>(a.xyzi, P, proj, range, key, n2b, bin_count, row_count, a.n_dev);
    ++launched;
  }
  k_bin_scan<<<n2b, kBinScanThreads, 0, st>>>(n2b, bin_count, row_count, bin_start, row_nxt, row_prv, sin_tab,
                                               hav_tab);
  ++launched;
  if (P > 0) {
    k_bin_scatter<<<(P + 255) / 256, 256, 0, st>>>(P, proj, key, bin_start, cursor, sorted, a.n_dev);
    ++launched;
  }
  const size_t q_threads = (size_t)a.n_queries * kGroup;
  k_nn_rows<<<(unsigned)((q_threads + kQueryThreads - 1) / kQueryThreads), kQueryThreads, 0, st>>>(
      n2b, a.grid, sorted, bin_start, row_nxt, row_prv, sin_tab, hav_tab, a.max_sq, a.xyzi, range, a.refl, a.amb,
      a.n_out_ch, a.out, a.nn_idx);
  ++launched;
  count_launches(launched);
  return cudaGetLastError();
}

}  // namespace phgpu
