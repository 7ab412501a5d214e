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
// Acceleration structure: points are bucketed on a 32^3 grid over
// [-1.0625, 1.0625]^3 ordered coarse-cell-major (8^3 coarse cells of 4^3 fine
// cells), with exact per-cell bounding boxes.  Cells are only pruned when
// their box lies beyond the current best distance (with a 1e-5 relative
// margin so float rounding can never prune the true nearest point), so the
// search is exact whatever bound it starts from.
//
// On the 2B x 2B Driscoll-Healy grid (k_nn_grid) the bound starts close to
// the answer: projection also drops every point into the grid's (theta, phi)
// bin and marks the bin in a per-phi-column row bitmask.  A direction takes
// the nearest occupied bins above and below it in its own and the two
// neighbouring columns on each side, plus every point of its own fine cell;
// far from the scanned band (most directions of a LiDAR scan) this lands
// within about one bin of the final distance.  Other direction sets
// (k_nn_query) start from one representative point per coarse cell.
#include "kernels.h"

namespace phgpu {

constexpr int kFineG = 32;
constexpr int kFineCells = kFineG * kFineG * kFineG;
constexpr int kCoarseG = 8;
constexpr int kCoarseCells = kCoarseG * kCoarseG * kCoarseG;
constexpr float kGridLo = -1.0625f;
constexpr float kGridInvH = 32.0f / 2.125f;

__device__ __forceinline__ int cell_coord(float v) {
  int c = (int)floorf((v - kGridLo) * kGridInvH);
  return min(max(c, 0), kFineG - 1);
}

__device__ __forceinline__ uint32_t cell_key(float x, float y, float z) {
  const int fx = cell_coord(x), fy = cell_coord(y), fz = cell_coord(z);
  const int cc = ((fz >> 2) * kCoarseG + (fy >> 2)) * kCoarseG + (fx >> 2);
  const int lf = ((fz & 3) * 4 + (fy & 3)) * 4 + (fx & 3);
  return (uint32_t)(cc * 64 + lf);
}

// float functions evaluated in double and rounded once (correctly rounded
// except in rare near-halfway cases; glibc's float versions can differ by one
// ulp, so projected coordinates match the reference with high probability).
__device__ __forceinline__ float acos_f(float x) { return (float)acos((double)x); }
__device__ __forceinline__ float atan2_f(float y, float x) { return (float)atan2((double)y, (double)x); }

// Bins of the 2B x 2B direction grid: row i covers theta in [i, i + 1) * pi / 2B,
// column j covers phi within pi / 2B of 2 pi j / 2B.  binmap[i * n2b + j] =
// lowest point index in the bin (init 0xffffffff), colmask[j * W + i / 32]
// bit i % 32 set when the bin is occupied (W = (n2b + 31) / 32).
__host__ __device__ __forceinline__ int bin_words(int n2b) { return (n2b + 31) >> 5; }

__global__ void k_project(const float4* __restrict__ xyzi, int P, float4* __restrict__ proj,
                          double* __restrict__ range, uint32_t* __restrict__ key,
                          uint32_t* __restrict__ cell_count, uint32_t* __restrict__ coarse_count, int n2b,
                          uint32_t* __restrict__ binmap, uint32_t* __restrict__ colmask) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P) return;
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
  const uint32_t k = cell_key(ox, oy, oz);
  key[i] = k;
  // consecutive points of a scan mostly share cells: one atomic per group of
  // lanes with the same key (a plain per-point atomic serialised on the
  // ~1000 points of a coarse cell)
  {
    const unsigned act = __activemask();
    const int lane = threadIdx.x & 31;
    const unsigned pf = __match_any_sync(act, k);
    if (lane == __ffs(pf) - 1) atomicAdd(&cell_count[k], (uint32_t)__popc(pf));
    const unsigned pc = __match_any_sync(act, k >> 6);
    if (lane == __ffs(pc) - 1) atomicAdd(&coarse_count[k >> 6], (uint32_t)__popc(pc));
  }
  if (n2b > 0) {
    const double w = M_PI / (double)n2b;  // bin height in theta, half bin width in phi
    const int bi = min(max((int)(tx / w), 0), n2b - 1);
    int bj = (int)floor(ty / (2.0 * w) + 0.5);
    bj = bj >= n2b ? bj - n2b : max(bj, 0);
    atomicMin(&binmap[bi * n2b + bj], (uint32_t)i);
    atomicOr(&colmask[bj * bin_words(n2b) + (bi >> 5)], 1u << (bi & 31));
  }
}

// Exclusive scan of the 32768 fine-cell counts and the compact list of
// non-empty coarse cells {start, count, coarse id} in coarse-id order: one
// 64-thread block per coarse cell (= its 64 fine cells) takes its base and
// list slot from the 512 coarse counts that precede it, then scans its own
// fine counts.
__global__ void __launch_bounds__(64) k_cell_scan(const uint32_t* __restrict__ count,
                                                  const uint32_t* __restrict__ coarse_count,
                                                  uint32_t* __restrict__ start, uint4* __restrict__ clist,
                                                  uint32_t* __restrict__ n_coarse) {
  __shared__ uint32_t s_pts[2], s_ne[2], s_fine[2];
  const int c = blockIdx.x, t = threadIdx.x, lane = t & 31, warp = t >> 5;
  uint32_t pts = 0, ne = 0;
  for (int i = t; i < c; i += 64) {
    const uint32_t v = __ldg(&coarse_count[i]);
    pts += v;
    ne += v > 0u ? 1u : 0u;
  }
  const uint32_t v = __ldg(&count[c * 64 + t]);
  uint32_t incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    pts += __shfl_xor_sync(0xffffffffu, pts, o);
    ne += __shfl_xor_sync(0xffffffffu, ne, o);
    const uint32_t u = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += u;
  }
  if (lane == 0) {
    s_pts[warp] = pts;
    s_ne[warp] = ne;
  }
  if (lane == 31) s_fine[warp] = incl;
  __syncthreads();
  const uint32_t base = s_pts[0] + s_pts[1], slot = s_ne[0] + s_ne[1];
  const uint32_t excl = incl - v + (warp ? s_fine[0] : 0u);
  start[c * 64 + t] = base + excl;
  if (t == 63) {
    const uint32_t total = excl + v;
    if (total > 0) clist[slot] = make_uint4(base, total, (uint32_t)c, 0u);
    if (c == kCoarseCells - 1) {
      start[kFineCells] = base + total;
      *n_coarse = slot + (total > 0 ? 1u : 0u);
    }
  }
}

__global__ void k_scatter(int P, const float4* __restrict__ proj, const uint32_t* __restrict__ key,
                          const uint32_t* __restrict__ start, uint32_t* __restrict__ cursor,
                          float4* __restrict__ sorted) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P) return;
  const uint32_t k = key[i];
  if (k == 0xffffffffu) return;
  const uint32_t slot = start[k] + atomicAdd(&cursor[k], 1u);
  const float4 p = proj[i];
  sorted[slot] = make_float4(p.x, p.y, p.z, __int_as_float(i));
}

__device__ __forceinline__ uint32_t ord(float v) { return float_order_bits(v); }

// Tight boxes of fine and coarse cells: thread per sorted point, warp-segmented
// min/max over lanes of the same cell, one atomic per segment.  Boxes hold
// order-preserving bits: lo[c*3+a] (init 0xffffffff), hi[c*3+a] (init 0).
__global__ void k_cell_bounds(const uint32_t* __restrict__ n_sorted, const float4* __restrict__ sorted,
                              uint32_t* __restrict__ flo, uint32_t* __restrict__ fhi, uint32_t* __restrict__ clo,
                              uint32_t* __restrict__ chi) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = i < (int)*n_sorted;
  float4 p = valid ? sorted[i] : make_float4(0.f, 0.f, 0.f, 0.f);
  const uint32_t fk = valid ? cell_key(p.x, p.y, p.z) : 0xffffffffu;
  const uint32_t v[3] = {ord(p.x), ord(p.y), ord(p.z)};
  // fine cell segments
  {
    const unsigned peers = __match_any_sync(0xffffffffu, fk);
    const int leader = __ffs(peers) - 1;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const uint32_t mn = __reduce_min_sync(peers, v[a]);
      const uint32_t mx = __reduce_max_sync(peers, v[a]);
      if (valid && (int)(threadIdx.x & 31) == leader) {
        atomicMin(&flo[fk * 3 + a], mn);
        atomicMax(&fhi[fk * 3 + a], mx);
      }
    }
  }
  // coarse cell segments
  {
    const uint32_t ck = valid ? fk >> 6 : 0xffffffffu;
    const unsigned peers = __match_any_sync(0xffffffffu, ck);
    const int leader = __ffs(peers) - 1;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const uint32_t mn = __reduce_min_sync(peers, v[a]);
      const uint32_t mx = __reduce_max_sync(peers, v[a]);
      if (valid && (int)(threadIdx.x & 31) == leader) {
        atomicMin(&clo[ck * 3 + a], mn);
        atomicMax(&chi[ck * 3 + a], mx);
      }
    }
  }
}

__device__ __forceinline__ float box_lb2(float qx, float qy, float qz, const float* b) {
  const float dx = fmaxf(fmaxf(b[0] - qx, qx - b[3]), 0.0f);
  const float dy = fmaxf(fmaxf(b[1] - qy, qy - b[4]), 0.0f);
  const float dz = fmaxf(fmaxf(b[2] - qz, qz - b[5]), 0.0f);
  return dx * dx + dy * dy + dz * dz;
}

__device__ __forceinline__ float box_lb2_ord(float qx, float qy, float qz, const uint32_t* lo,
                                             const uint32_t* hi) {
  float b[6];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    b[a] = float_from_order_bits(__ldg(&lo[a]));
    b[3 + a] = float_from_order_bits(__ldg(&hi[a]));
  }
  return box_lb2(qx, qy, qz, b);
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

__device__ __forceinline__ void warp_nn_min(float& best, int& bidx) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const float ob = __shfl_xor_sync(0xffffffffu, best, o);
    const int oi = __shfl_xor_sync(0xffffffffu, bidx, o);
    nn_update(ob, oi, best, bidx);
  }
}

constexpr int kQueryThreads = 256;
constexpr float kPruneMargin = 0.99999f;  // lower bound * margin must exceed the best to prune

// Best-first scan of one coarse cell: its non-empty fine cells are visited in
// ascending order of their box lower bound until the bound exceeds the best
// distance.  best / bidx are warp-uniform on entry and on exit.
__device__ __forceinline__ void scan_coarse(int cid, float qx, float qy, float qz,
                                            const float4* __restrict__ sorted,
                                            const uint32_t* __restrict__ fstart,
                                            const uint32_t* __restrict__ flo,
                                            const uint32_t* __restrict__ fhi, float& best, int& bidx) {
  const int lane = threadIdx.x & 31;
  float lb[2];
  uint32_t fs[2], fe[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int fc = cid * 64 + h * 32 + lane;
    fs[h] = __ldg(&fstart[fc]);
    fe[h] = __ldg(&fstart[fc + 1]);
    lb[h] = fe[h] > fs[h] ? box_lb2_ord(qx, qy, qz, flo + 3 * fc, fhi + 3 * fc) : INFINITY;
  }
  // at most 64 picks: every pick retires one fine cell
  for (int pick = 0; pick < 64; ++pick) {
    // warp argmin of the remaining lower bounds
    const int hsel = lb[1] < lb[0] ? 1 : 0;
    float m = lb[hsel];
    int who = lane * 2 + hsel;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const float om = __shfl_xor_sync(0xffffffffu, m, o);
      const int ow = __shfl_xor_sync(0xffffffffu, who, o);
      if (om < m || (om == m && ow < who)) {
        m = om;
        who = ow;
      }
    }
    if (!(m < INFINITY) || !(m * kPruneMargin <= best)) break;  // done, or nothing within the bound
    const int src = who >> 1, h = who & 1;
    const uint32_t s = __shfl_sync(0xffffffffu, h ? fs[1] : fs[0], src);
    const uint32_t e = __shfl_sync(0xffffffffu, h ? fe[1] : fe[0], src);
    if (lane == src) lb[h] = INFINITY;
    for (uint32_t j = s + lane; j < e; j += 32) {
      const float4 p = sorted[j];
      nn_update(ref_dist2(qx, qy, qz, p), __float_as_int(p.w), best, bidx);
    }
    warp_nn_min(best, bidx);
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

// One warp per grid direction (grid-stride).  The bound starts from one
// representative point per non-empty coarse cell; the coarse cell of the
// nearest representative is searched first, then every other coarse cell whose
// box lies within the bound.  Writes the sampled channels {range, intensity,
// reflectivity, ambient} (float) into out[ch][query] for ch < n_out_ch and the
// nearest index (or -1) into nn_idx.
__global__ void __launch_bounds__(kQueryThreads)
k_nn_query(int nq, const float4* __restrict__ grid, const float4* __restrict__ sorted,
           const uint32_t* __restrict__ fstart, const uint32_t* __restrict__ flo,
           const uint32_t* __restrict__ fhi, const uint4* __restrict__ clist,
           const uint32_t* __restrict__ clo, const uint32_t* __restrict__ chi,
           const uint32_t* __restrict__ n_coarse_p, float max_sq, const float4* __restrict__ xyzi,
           const double* __restrict__ range, const float* __restrict__ refl,
           const float* __restrict__ amb, int n_out_ch, float* __restrict__ out,
           int32_t* __restrict__ nn_idx) {
  __shared__ uint32_t s_cid[kCoarseCells];
  __shared__ float s_box[kCoarseCells * 6];
  __shared__ float4 s_rep[kCoarseCells];
  const int nc = (int)*n_coarse_p;
  for (int i = threadIdx.x; i < nc; i += blockDim.x) {
    const uint4 e = clist[i];
    s_cid[i] = e.z;
    s_rep[i] = sorted[e.x];
    for (int a = 0; a < 3; ++a) {
      s_box[6 * i + a] = float_from_order_bits(clo[e.z * 3 + a]);
      s_box[6 * i + 3 + a] = float_from_order_bits(chi[e.z * 3 + a]);
    }
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int wpb = blockDim.x >> 5;
  for (int qi = blockIdx.x * wpb + (threadIdx.x >> 5); qi < nq; qi += gridDim.x * wpb) {
    const float4 q = grid[qi];
    float best = INFINITY;
    int bidx = 0x7fffffff;
    // representatives: remember which coarse cell gave each lane's best
    int bcell = -1;
    for (int c = lane; c < nc; c += 32) {
      const float4 r = s_rep[c];
      const float d = ref_dist2(q.x, q.y, q.z, r);
      const int id = __float_as_int(r.w);
      if (d < best || (d == best && id < bidx)) {
        best = d;
        bidx = id;
        bcell = c;
      }
    }
    int first = bcell;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const float ob = __shfl_xor_sync(0xffffffffu, best, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bidx, o);
      const int oc = __shfl_xor_sync(0xffffffffu, first, o);
      if (ob < best || (ob == best && oi < bidx)) {
        best = ob;
        bidx = oi;
        first = oc;
      }
    }
    if (first >= 0) scan_coarse((int)s_cid[first], q.x, q.y, q.z, sorted, fstart, flo, fhi, best, bidx);
    for (int c0 = 0; c0 < nc; c0 += 32) {
      const int c = c0 + lane;
      const bool cand = c < nc && c != first && box_lb2(q.x, q.y, q.z, s_box + 6 * c) * kPruneMargin <= best;
      unsigned cmask = __ballot_sync(0xffffffffu, cand);
      while (cmask) {
        const int cc = c0 + __ffs(cmask) - 1;
        cmask &= cmask - 1;
        if (box_lb2(q.x, q.y, q.z, s_box + 6 * cc) * kPruneMargin > best) continue;  // warp-uniform
        scan_coarse((int)s_cid[cc], q.x, q.y, q.z, sorted, fstart, flo, fhi, best, bidx);
      }
    }
    if (lane == 0) emit_sample(qi, nq, best, bidx, max_sq, xyzi, range, refl, amb, n_out_ch, out, nn_idx);
  }
}

// Scans points [s, e) of the sorted array, four loads in flight per lane.
__device__ __forceinline__ void scan_points(uint32_t s, uint32_t e, float qx, float qy, float qz,
                                            const float4* __restrict__ sorted, float& best, int& bidx) {
  const int lane = threadIdx.x & 31;
  for (uint32_t j = s + lane; j < e; j += 128) {
    float4 p[4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (j + 32 * u < e) p[u] = sorted[j + 32 * u];
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (j + 32 * u < e) nn_update(ref_dist2(qx, qy, qz, p[u]), __float_as_int(p[u].w), best, bidx);
  }
}

// Nearest occupied row at or below (dir > 0) / above (dir < 0) row i in a
// column bitmask of W words; -1 when there is none.
__device__ __forceinline__ int nearest_row(const uint32_t* __restrict__ cm, int W, int i, int dir) {
  int w = i >> 5;
  const int b = i & 31;
  uint32_t m = __ldg(&cm[w]);
  if (dir > 0) {
    m &= 0xffffffffu << b;
    while (!m && ++w < W) m = __ldg(&cm[w]);
    return m ? (w << 5) + __ffs(m) - 1 : -1;
  }
  m &= b == 31 ? 0xffffffffu : ((1u << (b + 1)) - 1u);
  while (!m && --w >= 0) m = __ldg(&cm[w]);
  return m ? (w << 5) + 31 - __clz(m) : -1;
}

// One warp per direction of the 2B x 2B grid (grid-stride).  Bound: the
// points of the nearest occupied bins above and below in columns j-2..j+2
// (lanes 0..9), then all points of the direction's own fine cell; if no
// column near it holds any point, one representative per coarse cell.  Then
// every coarse cell whose box lies within the bound is opened and each of its
// fine cells within the bound is scanned; lanes keep private minima inside a
// coarse cell and the warp minimum (the bound for the next) is refreshed after it.
__global__ void __launch_bounds__(kQueryThreads)
k_nn_grid(int n2b, const float4* __restrict__ grid, const float4* __restrict__ proj,
          const uint32_t* __restrict__ binmap, const uint32_t* __restrict__ colmask,
          const float4* __restrict__ sorted, const uint32_t* __restrict__ fstart,
          const uint32_t* __restrict__ flo, const uint32_t* __restrict__ fhi, const uint4* __restrict__ clist,
          const uint32_t* __restrict__ clo, const uint32_t* __restrict__ chi,
          const uint32_t* __restrict__ n_coarse_p, float max_sq, const float4* __restrict__ xyzi,
          const double* __restrict__ range, const float* __restrict__ refl, const float* __restrict__ amb,
          int n_out_ch, float* __restrict__ out, int32_t* __restrict__ nn_idx) {
  __shared__ uint32_t s_cid[kCoarseCells];
  __shared__ float s_box[kCoarseCells * 6];
  __shared__ float4 s_rep[kCoarseCells];
  const int nc = (int)*n_coarse_p;
  for (int i = threadIdx.x; i < nc; i += blockDim.x) {
    const uint4 e = clist[i];
    s_cid[i] = e.z;
    s_rep[i] = sorted[e.x];
    for (int a = 0; a < 3; ++a) {
      s_box[6 * i + a] = float_from_order_bits(clo[e.z * 3 + a]);
      s_box[6 * i + 3 + a] = float_from_order_bits(chi[e.z * 3 + a]);
    }
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int wpb = blockDim.x >> 5;
  const int nq = n2b * n2b;
  const int W = bin_words(n2b);
  for (int qi = blockIdx.x * wpb + (threadIdx.x >> 5); qi < nq; qi += gridDim.x * wpb) {
    const float4 q = grid[qi];
    float best = INFINITY;
    int bidx = 0x7fffffff;
    if (lane < 10) {
      const int i = qi / n2b, j = qi - i * n2b;
      int jj = j + (lane >> 1) - 2;
      jj = jj < 0 ? jj + n2b : (jj >= n2b ? jj - n2b : jj);
      const int row = nearest_row(colmask + (size_t)jj * W, W, i, (lane & 1) ? 1 : -1);
      if (row >= 0) {
        const uint32_t sidx = __ldg(&binmap[row * n2b + jj]);
        nn_update(ref_dist2(q.x, q.y, q.z, __ldg(&proj[sidx])), (int)sidx, best, bidx);
      }
    }
    const uint32_t own = cell_key(q.x, q.y, q.z);
    scan_points(__ldg(&fstart[own]), __ldg(&fstart[own + 1]), q.x, q.y, q.z, sorted, best, bidx);
    warp_nn_min(best, bidx);
    if (!(best < INFINITY)) {
      for (int c = lane; c < nc; c += 32) {
        const float4 r = s_rep[c];
        nn_update(ref_dist2(q.x, q.y, q.z, r), __float_as_int(r.w), best, bidx);
      }
      warp_nn_min(best, bidx);
    }
    for (int c0 = 0; c0 < nc; c0 += 32) {
      const int c = c0 + lane;
      const bool cand = c < nc && box_lb2(q.x, q.y, q.z, s_box + 6 * c) * kPruneMargin <= best;
      unsigned cmask = __ballot_sync(0xffffffffu, cand);
      while (cmask) {
        const int cc = c0 + __ffs(cmask) - 1;
        cmask &= cmask - 1;
        const int cid = (int)s_cid[cc];
        uint32_t fs[2], fe[2];
        bool in[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const uint32_t fc = (uint32_t)(cid * 64 + h * 32 + lane);
          fs[h] = __ldg(&fstart[fc]);
          fe[h] = __ldg(&fstart[fc + 1]);
          in[h] = fe[h] > fs[h] && fc != own &&
                  box_lb2_ord(q.x, q.y, q.z, flo + 3 * fc, fhi + 3 * fc) * kPruneMargin <= best;
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          unsigned fmask = __ballot_sync(0xffffffffu, in[h]);
          while (fmask) {
            const int src = __ffs(fmask) - 1;
            fmask &= fmask - 1;
            const uint32_t s1 = __shfl_sync(0xffffffffu, fs[h], src);
            const uint32_t e1 = __shfl_sync(0xffffffffu, fe[h], src);
            scan_points(s1, e1, q.x, q.y, q.z, sorted, best, bidx);
          }
        }
        warp_nn_min(best, bidx);
      }
    }
    if (lane == 0) emit_sample(qi, nq, best, bidx, max_sq, xyzi, range, refl, amb, n_out_ch, out, nn_idx);
  }
}

// ---------------------------------------------------------------- launcher

std::atomic<unsigned long long> g_launch_count{0};

size_t sampler_scratch_bytes(int max_points, int max_queries) {
  size_t b = (size_t)max_queries * sizeof(uint32_t) * 2;  // bin map + column masks (<= one word per bin)
  b += (size_t)max_points * sizeof(float4);    // proj
  b += (size_t)max_points * sizeof(double);    // range
  b += (size_t)max_points * sizeof(uint32_t);  // key
  b += (size_t)max_points * sizeof(float4);    // sorted
  b += (size_t)kFineCells * sizeof(uint32_t) * 2;   // count, cursor
  b += (size_t)kCoarseCells * sizeof(uint32_t);      // coarse counts
  b += (size_t)(kFineCells + 4) * sizeof(uint32_t);  // start
  b += (size_t)kFineCells * 6 * sizeof(uint32_t);    // fine boxes
  b += (size_t)kCoarseCells * sizeof(uint4);
  b += (size_t)kCoarseCells * 6 * sizeof(uint32_t);
  b += 256;
  return b + 20 * 256;  // carve() rounds each of the regions up to 256 bytes
}

static inline char* carve(char*& p, size_t bytes) {
  char* r = p;
  p += (bytes + 255) & ~(size_t)255;
  return r;
}

cudaError_t launch_sample(const SampleArgs& a, cudaStream_t st) {
  char* p = (char*)a.scratch;
  float4* proj = (float4*)carve(p, (size_t)a.max_points * sizeof(float4));
  double* range = (double*)carve(p, (size_t)a.max_points * sizeof(double));
  uint32_t* key = (uint32_t*)carve(p, (size_t)a.max_points * sizeof(uint32_t));
  float4* sorted = (float4*)carve(p, (size_t)a.max_points * sizeof(float4));
  uint32_t* count = (uint32_t*)carve(p, (size_t)kFineCells * sizeof(uint32_t));
  uint32_t* cursor = (uint32_t*)carve(p, (size_t)kFineCells * sizeof(uint32_t));
  uint32_t* ccount = (uint32_t*)carve(p, (size_t)kCoarseCells * sizeof(uint32_t));
  uint32_t* start = (uint32_t*)carve(p, (size_t)(kFineCells + 4) * sizeof(uint32_t));
  uint32_t* flo = (uint32_t*)carve(p, (size_t)kFineCells * 3 * sizeof(uint32_t));
  uint32_t* fhi = (uint32_t*)carve(p, (size_t)kFineCells * 3 * sizeof(uint32_t));
  uint4* clist = (uint4*)carve(p, (size_t)kCoarseCells * sizeof(uint4));
  uint32_t* clo = (uint32_t*)carve(p, (size_t)kCoarseCells * 3 * sizeof(uint32_t));
  uint32_t* chi = (uint32_t*)carve(p, (size_t)kCoarseCells * 3 * sizeof(uint32_t));
  uint32_t* ncoarse = (uint32_t*)carve(p, 256);
  const int n2b = a.n2b;
  const size_t nbins = (size_t)n2b * n2b, nmask = (size_t)n2b * bin_words(n2b);
  uint32_t* binmap = (uint32_t*)carve(p, nbins * sizeof(uint32_t));
  uint32_t* colmask = (uint32_t*)carve(p, nmask * sizeof(uint32_t));

  // count, cursor and coarse counts are adjacent: one memset
  cudaMemsetAsync(count, 0, (size_t)(2 * kFineCells + kCoarseCells) * sizeof(uint32_t), st);
  cudaMemsetAsync(flo, 0xff, (size_t)kFineCells * 3 * sizeof(uint32_t), st);
  cudaMemsetAsync(fhi, 0, (size_t)kFineCells * 3 * sizeof(uint32_t), st);
  cudaMemsetAsync(clo, 0xff, (size_t)kCoarseCells * 3 * sizeof(uint32_t), st);
  cudaMemsetAsync(chi, 0, (size_t)kCoarseCells * 3 * sizeof(uint32_t), st);
  if (n2b > 0) {
    cudaMemsetAsync(binmap, 0xff, nbins * sizeof(uint32_t), st);
    cudaMemsetAsync(colmask, 0, nmask * sizeof(uint32_t), st);
  }
  const int P = a.n_points;
  int launched = 0;
  if (P > 0) {
    k_project<<<(P + 255) / 256, 256, 0, st>>>(a.xyzi, P, proj, range, key, count, ccount, n2b, binmap, colmask);
    ++launched;
  }
  k_cell_scan<<<kCoarseCells, 64, 0, st>>>(count, ccount, start, clist, ncoarse);
  ++launched;
  if (P > 0) {
    k_scatter<<<(P + 255) / 256, 256, 0, st>>>(P, proj, key, start, cursor, sorted);
    k_cell_bounds<<<(P + 255) / 256, 256, 0, st>>>(start + kFineCells, sorted, flo, fhi, clo, chi);
    launched += 2;
  }
  const int wpb = kQueryThreads / 32;
  int blocks = (a.n_queries + wpb - 1) / wpb;
  if (blocks > 148 * 8) blocks = 148 * 8;
  if (n2b > 0) {
    k_nn_grid<<<blocks, kQueryThreads, 0, st>>>(n2b, a.grid, proj, binmap, colmask, sorted, start, flo, fhi, clist,
                                                clo, chi, ncoarse, a.max_sq, a.xyzi, range, a.refl, a.amb,
                                                a.n_out_ch, a.out, a.nn_idx);
  } else {
    k_nn_query<<<blocks, kQueryThreads, 0, st>>>(a.n_queries, a.grid, sorted, start, flo, fhi, clist, clo, chi,
                                                 ncoarse, a.max_sq, a.xyzi, range, a.refl, a.amb, a.n_out_ch,
                                                 a.out, a.nn_idx);
  }
  ++launched;
  count_launches(launched);
  return cudaGetLastError();
}

}  // namespace phgpu
