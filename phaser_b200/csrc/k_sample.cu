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
// cells); every non-empty coarse cell carries its exact box and a compact list
// of records {exact box, point range} of its non-empty fine cells.  Cells are only pruned when
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

// Cell records.  For list entry i (non-empty coarse cell clist[i].z) the
// non-empty fine cells are records frec[2 (64 i + j)], frec[2 (64 i + j) + 1],
// j < nfine[i], in fine-id order:
//   {lo.x, lo.y, lo.z, hi.x}, {hi.y, hi.z, start (bits), end (bits)}
// and the coarse box is cbox[2 i], cbox[2 i + 1] = {lo.xyz, hi.x}, {hi.yz, nfine (bits), 0}.
// One block per list entry: warps take fine cells, lanes the cell's points.
constexpr int kRecordThreads = 256;

__global__ void __launch_bounds__(kRecordThreads)
k_cell_records(const uint4* __restrict__ clist, const uint32_t* __restrict__ n_coarse_p,
               const uint32_t* __restrict__ fstart, const float4* __restrict__ sorted, float4* __restrict__ frec,
               float4* __restrict__ cbox) {
  __shared__ int s_fid[64];
  __shared__ int s_nf;
  __shared__ float s_box[kRecordThreads / 32][6];
  const int i = blockIdx.x;
  if (i >= (int)*n_coarse_p) return;
  const int c = (int)clist[i].z;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  if (warp == 0) {  // compact the non-empty fine cells of this coarse cell
    int base = 0;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int fc = c * 64 + h * 32 + lane;
      const bool ne = __ldg(&fstart[fc + 1]) > __ldg(&fstart[fc]);
      const unsigned m = __ballot_sync(0xffffffffu, ne);
      if (ne) s_fid[base + __popc(m & ((1u << lane) - 1u))] = fc;
      base += __popc(m);
    }
    if (lane == 0) s_nf = base;
  }
  __syncthreads();
  const int nf = s_nf;
  float wb[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
  for (int j = warp; j < nf; j += kRecordThreads / 32) {
    const int fc = s_fid[j];
    const uint32_t ps = __ldg(&fstart[fc]), pe = __ldg(&fstart[fc + 1]);
    float b[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
    for (uint32_t k = ps + lane; k < pe; k += 32) {
      const float4 p = sorted[k];
      b[0] = fminf(b[0], p.x);
      b[1] = fminf(b[1], p.y);
      b[2] = fminf(b[2], p.z);
      b[3] = fmaxf(b[3], p.x);
      b[4] = fmaxf(b[4], p.y);
      b[5] = fmaxf(b[5], p.z);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        b[a] = fminf(b[a], __shfl_xor_sync(0xffffffffu, b[a], o));
        b[3 + a] = fmaxf(b[3 + a], __shfl_xor_sync(0xffffffffu, b[3 + a], o));
      }
    }
    if (lane == 0) {
      float4* r = frec + 2 * ((size_t)i * 64 + j);
      r[0] = make_float4(b[0], b[1], b[2], b[3]);
      r[1] = make_float4(b[4], b[5], __uint_as_float(ps), __uint_as_float(pe));
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      wb[a] = fminf(wb[a], b[a]);
      wb[3 + a] = fmaxf(wb[3 + a], b[3 + a]);
    }
  }
  if (lane == 0) {
#pragma unroll
    for (int a = 0; a < 6; ++a) s_box[warp][a] = wb[a];
  }
  __syncthreads();
  if (t == 0) {
    float cb[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
    for (int w = 0; w < kRecordThreads / 32; ++w) {
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        cb[a] = fminf(cb[a], s_box[w][a]);
        cb[3 + a] = fmaxf(cb[3 + a], s_box[w][3 + a]);
      }
    }
    cbox[2 * i] = make_float4(cb[0], cb[1], cb[2], cb[3]);
    cbox[2 * i + 1] = make_float4(cb[4], cb[5], __int_as_float(nf), 0.f);
  }
}

__device__ __forceinline__ float box_lb2(float qx, float qy, float qz, const float* b) {
  const float dx = fmaxf(fmaxf(b[0] - qx, qx - b[3]), 0.0f);
  const float dy = fmaxf(fmaxf(b[1] - qy, qy - b[4]), 0.0f);
  const float dz = fmaxf(fmaxf(b[2] - qz, qz - b[5]), 0.0f);
  return dx * dx + dy * dy + dz * dz;
}

// Squared distance from q to a record's box; the record's point range in s, e.
__device__ __forceinline__ float rec_lb2(float qx, float qy, float qz, const float4* __restrict__ r, uint32_t& s,
                                         uint32_t& e) {
  const float4 a = __ldg(&r[0]), b = __ldg(&r[1]);
  s = __float_as_uint(b.z);
  e = __float_as_uint(b.w);
  const float dx = fmaxf(fmaxf(a.x - qx, qx - a.w), 0.0f);
  const float dy = fmaxf(fmaxf(a.y - qy, qy - b.x), 0.0f);
  const float dz = fmaxf(fmaxf(a.z - qz, qz - b.y), 0.0f);
  return dx * dx + dy * dy + dz * dz;
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

// Opens coarse list entry cc: every fine record within the bound (except the
// one starting at skip_start) is scanned; lanes keep private minima, the warp
// minimum is taken at the end.  best / bidx are warp-uniform on entry and exit.
__device__ __forceinline__ void open_coarse(int cc, int nf, uint32_t skip_start, float qx, float qy, float qz,
                                            const float4* __restrict__ frec, const float4* __restrict__ sorted,
                                            float& best, int& bidx) {
  const int lane = threadIdx.x & 31;
  const float bound = best;
  for (int j0 = 0; j0 < nf; j0 += 32) {
    const int j = j0 + lane;
    uint32_t s = 0, e = 0;
    bool in = false;
    if (j < nf) {
      const float lb = rec_lb2(qx, qy, qz, frec + 2 * ((size_t)cc * 64 + j), s, e);
      in = s != skip_start && lb * kPruneMargin <= bound;
    }
    unsigned m = __ballot_sync(0xffffffffu, in);
    while (m) {
      const int src = __ffs(m) - 1;
      m &= m - 1;
      scan_points(__shfl_sync(0xffffffffu, s, src), __shfl_sync(0xffffffffu, e, src), qx, qy, qz, sorted, best,
                  bidx);
    }
  }
  warp_nn_min(best, bidx);
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

// Shared prologue of the query kernels: coarse boxes, fine-record counts and
// one representative point per non-empty coarse cell.
struct CoarseSmem {
  float box[kCoarseCells * 6];
  int nf[kCoarseCells];
  float4 rep[kCoarseCells];
};

__device__ __forceinline__ int load_coarse(CoarseSmem& cs, const uint4* __restrict__ clist,
                                           const float4* __restrict__ cbox, const uint32_t* __restrict__ n_coarse_p,
                                           const float4* __restrict__ sorted) {
  const int nc = (int)*n_coarse_p;
  for (int i = threadIdx.x; i < nc; i += blockDim.x) {
    const float4 a = cbox[2 * i], b = cbox[2 * i + 1];
    cs.box[6 * i + 0] = a.x;
    cs.box[6 * i + 1] = a.y;
    cs.box[6 * i + 2] = a.z;
    cs.box[6 * i + 3] = a.w;
    cs.box[6 * i + 4] = b.x;
    cs.box[6 * i + 5] = b.y;
    cs.nf[i] = __float_as_int(b.z);
    cs.rep[i] = sorted[clist[i].x];
  }
  __syncthreads();
  return nc;
}

// Bound from the representatives (lane-parallel), then every coarse cell
// whose box lies within the bound is opened.
__device__ __forceinline__ void rep_bound(const CoarseSmem& cs, int nc, float qx, float qy, float qz, float& best,
                                          int& bidx) {
  const int lane = threadIdx.x & 31;
  for (int c = lane; c < nc; c += 32) {
    const float4 r = cs.rep[c];
    nn_update(ref_dist2(qx, qy, qz, r), __float_as_int(r.w), best, bidx);
  }
  warp_nn_min(best, bidx);
}

__device__ __forceinline__ void open_within(const CoarseSmem& cs, int nc, uint32_t skip_start, float qx, float qy,
                                            float qz, const float4* __restrict__ frec,
                                            const float4* __restrict__ sorted, float& best, int& bidx) {
  const int lane = threadIdx.x & 31;
  for (int c0 = 0; c0 < nc; c0 += 32) {
    const int c = c0 + lane;
    const bool cand = c < nc && box_lb2(qx, qy, qz, cs.box + 6 * c) * kPruneMargin <= best;
    unsigned cmask = __ballot_sync(0xffffffffu, cand);
    while (cmask) {
      const int cc = c0 + __ffs(cmask) - 1;
      cmask &= cmask - 1;
      if (box_lb2(qx, qy, qz, cs.box + 6 * cc) * kPruneMargin > best) continue;  // warp-uniform
      open_coarse(cc, cs.nf[cc], skip_start, qx, qy, qz, frec, sorted, best, bidx);
    }
  }
}

// One warp per direction of an arbitrary set (grid-stride): bound from the
// representatives, then the coarse cells within it.
__global__ void __launch_bounds__(kQueryThreads)
k_nn_query(int nq, const float4* __restrict__ grid, const float4* __restrict__ sorted,
           const float4* __restrict__ frec, const uint4* __restrict__ clist, const float4* __restrict__ cbox,
           const uint32_t* __restrict__ n_coarse_p, float max_sq, const float4* __restrict__ xyzi,
           const double* __restrict__ range, const float* __restrict__ refl, const float* __restrict__ amb,
           int n_out_ch, float* __restrict__ out, int32_t* __restrict__ nn_idx) {
  __shared__ CoarseSmem cs;
  const int nc = load_coarse(cs, clist, cbox, n_coarse_p, sorted);
  const int lane = threadIdx.x & 31;
  const int wpb = blockDim.x >> 5;
  for (int qi = blockIdx.x * wpb + (threadIdx.x >> 5); qi < nq; qi += gridDim.x * wpb) {
    const float4 q = grid[qi];
    float best = INFINITY;
    int bidx = 0x7fffffff;
    rep_bound(cs, nc, q.x, q.y, q.z, best, bidx);
    open_within(cs, nc, 0xffffffffu, q.x, q.y, q.z, frec, sorted, best, bidx);
    if (lane == 0) emit_sample(qi, nq, best, bidx, max_sq, xyzi, range, refl, amb, n_out_ch, out, nn_idx);
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
// every coarse cell whose box lies within the bound is opened.
__global__ void __launch_bounds__(kQueryThreads)
k_nn_grid(int n2b, const float4* __restrict__ grid, const float4* __restrict__ proj,
          const uint32_t* __restrict__ binmap, const uint32_t* __restrict__ colmask,
          const float4* __restrict__ sorted, const uint32_t* __restrict__ fstart, const float4* __restrict__ frec,
          const uint4* __restrict__ clist, const float4* __restrict__ cbox, const uint32_t* __restrict__ n_coarse_p,
          float max_sq, const float4* __restrict__ xyzi, const double* __restrict__ range,
          const float* __restrict__ refl, const float* __restrict__ amb, int n_out_ch, float* __restrict__ out,
          int32_t* __restrict__ nn_idx) {
  __shared__ CoarseSmem cs;
  const int nc = load_coarse(cs, clist, cbox, n_coarse_p, sorted);
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
    const uint32_t own_s = __ldg(&fstart[own]), own_e = __ldg(&fstart[own + 1]);
    scan_points(own_s, own_e, q.x, q.y, q.z, sorted, best, bidx);
    warp_nn_min(best, bidx);
    if (!(best < INFINITY)) rep_bound(cs, nc, q.x, q.y, q.z, best, bidx);
    open_within(cs, nc, own_e > own_s ? own_s : 0xffffffffu, q.x, q.y, q.z, frec, sorted, best, bidx);
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
  b += (size_t)kFineCells * 2 * sizeof(float4);      // fine records
  b += (size_t)kCoarseCells * sizeof(uint4);         // coarse list
  b += (size_t)kCoarseCells * 2 * sizeof(float4);    // coarse boxes
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
  float4* frec = (float4*)carve(p, (size_t)kFineCells * 2 * sizeof(float4));
  uint4* clist = (uint4*)carve(p, (size_t)kCoarseCells * sizeof(uint4));
  float4* cbox = (float4*)carve(p, (size_t)kCoarseCells * 2 * sizeof(float4));
  uint32_t* ncoarse = (uint32_t*)carve(p, 256);
  const int n2b = a.n2b;
  const size_t nbins = (size_t)n2b * n2b, nmask = (size_t)n2b * bin_words(n2b);
  uint32_t* binmap = (uint32_t*)carve(p, nbins * sizeof(uint32_t));
  uint32_t* colmask = (uint32_t*)carve(p, nmask * sizeof(uint32_t));

  // count, cursor and coarse counts are adjacent: one memset
  cudaMemsetAsync(count, 0, (size_t)(2 * kFineCells + kCoarseCells) * sizeof(uint32_t), st);
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
    k_cell_records<<<kCoarseCells, kRecordThreads, 0, st>>>(clist, ncoarse, start, sorted, frec, cbox);
    launched += 2;
  }
  const int wpb = kQueryThreads / 32;
  int blocks = (a.n_queries + wpb - 1) / wpb;
  if (blocks > 148 * 8) blocks = 148 * 8;
  if (n2b > 0) {
    k_nn_grid<<<blocks, kQueryThreads, 0, st>>>(n2b, a.grid, proj, binmap, colmask, sorted, start, frec, clist, cbox,
                                                ncoarse, a.max_sq, a.xyzi, range, a.refl, a.amb, a.n_out_ch, a.out,
                                                a.nn_idx);
  } else {
    k_nn_query<<<blocks, kQueryThreads, 0, st>>>(a.n_queries, a.grid, sorted, frec, clist, cbox, ncoarse, a.max_sq,
                                                 a.xyzi, range, a.refl, a.amb, a.n_out_ch, a.out, a.nn_idx);
  }
  ++launched;
  count_launches(launched);
  return cudaGetLastError();
}

}  // namespace phgpu
