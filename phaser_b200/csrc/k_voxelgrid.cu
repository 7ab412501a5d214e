// Voxel-grid downsampling on the GPU: preproc::VoxelGridCmd
// (phaser_pre/src/commands/voxel-grid-cmd.cc:11-22), which runs
// pcl::VoxelGrid<pcl::PointXYZI> (PCL 1.8.1, the libpcl-dev of the
// reference's Ubuntu 18.04 / ROS Melodic image; PCL is not part of the
// reference tree) with leaf --phaser_voxel_grid_leaf_size (0.25) in place.
//
// pcl::VoxelGrid::applyFilter, restated:
//   * min/max of x, y, z over the finite points (getMinMax3D);
//   * inv = 1 / leaf (float); d = int64((max - min) * inv) + 1 per axis; if
//     dx*dy*dz > INT32_MAX the output is the input (an overflow warning);
//   * min_b = int(floor(min * inv)), max_b = int(floor(max * inv)),
//     div_b = max_b - min_b + 1, multipliers (1, div_x, div_x * div_y);
//   * per finite point: ijk = int(floor(p * inv) - float(min_b)) per axis and
//     leaf index = ijk . multipliers (x fastest);
//   * sort the (leaf, point) pairs by leaf; every run of one leaf with at least
//     min_points_per_voxel points becomes one output point, the float sum of
//     x, y, z, intensity over the run divided by float(run length); leaves
//     come out in increasing leaf index.
// PCL sorts with std::sort, whose order among the points of one leaf is
// unspecified; here the sort is stable, so a leaf's points are summed in
// input order, which fixes the result bit for bit (the oracle sums in the
// same order).  Non-finite points are dropped (PCL does so for clouds flagged
// not dense and is undefined otherwise).  Leaf grids whose indices leave
// int32 (|floor(coordinate / leaf)| >= 2^31), with more than 2^30 leaves along
// an axis, or whose cell count leaves 32 bits are refused with
// PHGPU_ERR_LIMIT: PCL's int arithmetic is undefined there.
//
// GPU layout: every step is a pass over 32-bit words in HBM -- a bounds
// reduction, a stable compaction of the finite points into (leaf, point)
// pairs, four stable 8-bit LSD radix passes (per-tile digit counts, a
// per-digit scan over tiles, a ranked scatter), a compaction of the leaf
// heads, and one warp per leaf for the centroid (gathers pipelined two
// batches ahead, in-order float sums).
// Nothing synchronises the host until the output count is read.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <string>

#include "../../include/phaser_gpu.h"
#include "kernels.h"

namespace phgpu {
namespace {

constexpr int kVgThreads = 256;
constexpr int kVgWarps = kVgThreads / 32;
constexpr int kVgRounds = 8;
constexpr int kVgTile = kVgThreads * kVgRounds;  // items per block and pass
constexpr int kBins = 256;                        // 8-bit radix digits
constexpr int kScanThreads = 1024;

enum VgStatus : int32_t { kVgOk = 0, kVgEmpty = 1, kVgOverflow = 2, kVgRange = 3 };

struct VgState {
  uint32_t lo_inv[3];  // max of ~order(x): decodes to the minimum
  uint32_t hi[3];      // max of order(x); 0 = no finite point
  int32_t status;
  int32_t min_b[3];
  uint32_t mul[3];
  uint32_t n_valid;   // finite points
  uint32_t n_leaves;  // occupied leaves
  uint32_t n_out;     // leaves kept (>= min points)
};

__device__ __forceinline__ bool finite3(float4 p) { return isfinite(p.x) && isfinite(p.y) && isfinite(p.z); }

__device__ __forceinline__ uint32_t lanemask_lt() { return (1u << (threadIdx.x & 31)) - 1u; }

// ---------------------------------------------------------------- bounds
// Per block: max of ~order(v) (decodes to the minimum) and of order(v) per
// axis over the finite points, written to part[block][6]; k_vg_plan reduces
// the blocks (no atomics on a few hot words).
constexpr int kBoundsBlocks = 148 * 4;

__global__ void __launch_bounds__(kVgThreads) k_vg_bounds(const float4* __restrict__ pts, uint32_t n,
                                                          uint32_t* __restrict__ part) {
  uint32_t m[6] = {0, 0, 0, 0, 0, 0};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float4 p = pts[i];
    if (!finite3(p)) continue;
    const float v[3] = {p.x, p.y, p.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const uint32_t o = float_order_bits(v[a]);
      m[a] = max(m[a], ~o);
      m[3 + a] = max(m[3 + a], o);
    }
  }
  __shared__ uint32_t s_m[kVgWarps][6];
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    for (int off = 16; off > 0; off >>= 1) m[c] = max(m[c], __shfl_xor_sync(0xffffffffu, m[c], off));
    if ((threadIdx.x & 31) == 0) s_m[threadIdx.x >> 5][c] = m[c];
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    uint32_t r = 0;
    for (int w = 0; w < kVgWarps; ++w) r = max(r, s_m[w][threadIdx.x]);
    part[blockIdx.x * 6 + threadIdx.x] = r;
  }
}

// ---------------------------------------------------------------- plan
// Reduces the bounds partials (one warp), then lane 0 plans the grid.
__global__ void k_vg_plan(const uint32_t* __restrict__ part, int n_part, VgState* st, float inv_x, float inv_y,
                          float inv_z) {
  const int lane = threadIdx.x & 31;
  uint32_t m[6] = {0, 0, 0, 0, 0, 0};
  for (int b = lane; b < n_part; b += 32)
    for (int c = 0; c < 6; ++c) m[c] = max(m[c], part[b * 6 + c]);
  for (int c = 0; c < 6; ++c)
    for (int off = 16; off > 0; off >>= 1) m[c] = max(m[c], __shfl_xor_sync(0xffffffffu, m[c], off));
  if (threadIdx.x != 0) return;
  for (int a = 0; a < 3; ++a) {
    st->lo_inv[a] = m[a];
    st->hi[a] = m[3 + a];
  }
  st->n_valid = st->n_leaves = st->n_out = 0;
  if (st->hi[0] == 0) {
    st->status = kVgEmpty;
    return;
  }
  const float inv[3] = {inv_x, inv_y, inv_z};
  float mn[3], mx[3];
  long long d[3], div[3];
  bool overflow = false, range = false;
  for (int a = 0; a < 3; ++a) {
    mn[a] = float_from_order_bits(~st->lo_inv[a]);
    mx[a] = float_from_order_bits(st->hi[a]);
    const float ext = __fmul_rn(__fsub_rn(mx[a], mn[a]), inv[a]);
    if (!(ext < 4.0e18f)) {  // the int64 conversion itself would overflow
      overflow = true;
      d[a] = 0;
    } else {
      d[a] = (long long)ext + 1;
    }
    const float fb_lo = floorf(__fmul_rn(mn[a], inv[a]));
    const float fb_hi = floorf(__fmul_rn(mx[a], inv[a]));
    if (!(fb_lo >= -2147483648.0f && fb_hi < 2147483648.0f)) range = true;
    st->min_b[a] = range ? 0 : (int32_t)fb_lo;
    div[a] = range ? 1 : (long long)(int32_t)fb_hi - (long long)(int32_t)fb_lo + 1;
    // ijk = float(floor) - float(min_b) must convert to int exactly
    if (div[a] > (1ll << 30)) range = true;
  }
  if (!overflow) {
    // dx * dy * dz > INT32_MAX, evaluated without int64 overflow
    if (d[0] > 2147483647ll || d[1] > 2147483647ll || d[2] > 2147483647ll) overflow = true;
    else if (d[0] * d[1] > 2147483647ll) overflow = true;
    else overflow = d[0] * d[1] * d[2] > 2147483647ll;
  }
  if (overflow) {
    st->status = kVgOverflow;
    return;
  }
  const unsigned long long cells = (unsigned long long)div[0] * (unsigned long long)div[1] * (unsigned long long)div[2];
  if (range || cells > 0xffffffffull) {
    st->status = kVgRange;
    return;
  }
  st->mul[0] = 1u;
  st->mul[1] = (uint32_t)div[0];
  st->mul[2] = (uint32_t)div[0] * (uint32_t)div[1];
  st->status = kVgOk;
}

// ---------------------------------------------------------------- scan
// Exclusive scan of `len` words by one block; *total gets the sum.
__global__ void __launch_bounds__(kScanThreads) k_scan_words(const uint32_t* __restrict__ in, uint32_t len,
                                                             uint32_t* __restrict__ out, uint32_t* total) {
  __shared__ uint32_t s_warp[kScanThreads / 32];
  const uint32_t chunk = (len + kScanThreads - 1) / kScanThreads;
  const uint32_t b = threadIdx.x * chunk;
  const uint32_t e = min(len, b + chunk);
  uint32_t sum = 0;
  for (uint32_t i = b; i < e; ++i) sum += in[i];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t incl = sum;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) s_warp[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = s_warp[lane];
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t v = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += v;
    }
    s_warp[lane] = w;  // inclusive over warps
  }
  __syncthreads();
  uint32_t run = incl - sum + (warp > 0 ? s_warp[warp - 1] : 0u);
  for (uint32_t i = b; i < e; ++i) {
    const uint32_t v = in[i];
    out[i] = run;
    run += v;
  }
  if (threadIdx.x == kScanThreads - 1 && total) *total = run;
}

// ---------------------------------------------------------------- stable compaction
// Op: __device__ uint32_t n() const; bool flag(uint32_t i) const (i < n());
//     void emit(uint32_t i, uint32_t pos) const.  Item order inside a tile
//     is (round, thread), i.e. ascending index, so ranks are stable.
template <class Op>
__global__ void __launch_bounds__(kVgThreads) k_flag_count(Op op, uint32_t* __restrict__ counts) {
  const uint32_t n = op.n();
  const uint32_t base = blockIdx.x * kVgTile;
  bool f[kVgRounds];  // all of the tile's flags first: one load latency, not one per round
#pragma unroll
  for (int r = 0; r < kVgRounds; ++r) {
    const uint32_t i = base + r * kVgThreads + threadIdx.x;
    f[r] = i < n && op.flag(i);
  }
  uint32_t c = 0;
#pragma unroll
  for (int r = 0; r < kVgRounds; ++r) c += __popc(__ballot_sync(0xffffffffu, f[r]));
  __shared__ uint32_t s[kVgWarps];
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int w = 0; w < kVgWarps; ++w) t += s[w];
    counts[blockIdx.x] = t;
  }
}

template <class Op>
__global__ void __launch_bounds__(kVgThreads) k_flag_scatter(Op op, const uint32_t* __restrict__ offsets) {
  const uint32_t n = op.n();
  const uint32_t base = blockIdx.x * kVgTile;
  if (base >= n) return;
  __shared__ uint32_t s_w[kVgWarps];
  const int warp = threadIdx.x >> 5;
  uint32_t run = offsets[blockIdx.x];
  bool fl[kVgRounds];
#pragma unroll
  for (int r = 0; r < kVgRounds; ++r) {
    const uint32_t i = base + r * kVgThreads + threadIdx.x;
    fl[r] = i < n && op.flag(i);
  }
#pragma unroll
  for (int r = 0; r < kVgRounds; ++r) {
    const uint32_t i = base + r * kVgThreads + threadIdx.x;
    const bool f = fl[r];
    const uint32_t bal = __ballot_sync(0xffffffffu, f);
    if ((threadIdx.x & 31) == 0) s_w[warp] = __popc(bal);
    __syncthreads();
    uint32_t before = 0, all = 0;
    for (int w = 0; w < kVgWarps; ++w) {
      const uint32_t c = s_w[w];
      before += w < warp ? c : 0u;
      all += c;
    }
    if (f) op.emit(i, run + before + __popc(bal & lanemask_lt()));
    run += all;
    __syncthreads();
  }
}

// Finite points -> (leaf, point) pairs in input order.
struct ValidOp {
  const float4* pts;
  uint32_t n_points;
  float inv[3];
  const VgState* st;
  uint32_t* keys;
  uint32_t* vals;
  __device__ uint32_t n() const { return st->status == kVgOk ? n_points : 0u; }
  __device__ bool flag(uint32_t i) const { return finite3(pts[i]); }
  __device__ void emit(uint32_t i, uint32_t pos) const {
    const float4 p = pts[i];
    const float v[3] = {p.x, p.y, p.z};
    uint32_t key = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float f = floorf(__fmul_rn(v[a], inv[a]));
      const int32_t ijk = (int32_t)__fsub_rn(f, (float)st->min_b[a]);
      key += (uint32_t)ijk * st->mul[a];
    }
    keys[pos] = key;
    vals[pos] = i;
  }
};

// First entry of every run of one leaf in the sorted pairs.
struct HeadOp {
  const uint32_t* keys;
  const VgState* st;
  uint32_t* leaf_start;
  __device__ uint32_t n() const { return st->n_valid; }
  __device__ bool flag(uint32_t i) const { return i == 0 || keys[i] != keys[i - 1]; }
  __device__ void emit(uint32_t i, uint32_t pos) const { leaf_start[pos] = i; }
};

// Leaves with at least min_points points (centroids staged per leaf).
struct KeepOp {
  const uint32_t* leaf_start;
  const VgState* st;
  uint32_t min_points;
  const float4* tmp;
  const float* tmp_refl;
  const float* tmp_amb;
  float4* out;
  float* out_refl;
  float* out_amb;
  __device__ uint32_t n() const { return st->n_leaves; }
  __device__ bool flag(uint32_t j) const {
    const uint32_t e = j + 1 < st->n_leaves ? leaf_start[j + 1] : st->n_valid;
    return e - leaf_start[j] >= min_points;
  }
  __device__ void emit(uint32_t j, uint32_t pos) const {
    out[pos] = tmp[j];
    if (out_refl) out_refl[pos] = tmp_refl[j];
    if (out_amb) out_amb[pos] = tmp_amb[j];
  }
};

// ---------------------------------------------------------------- radix passes
__global__ void __launch_bounds__(kVgThreads) k_radix_count(const uint32_t* __restrict__ keys, const VgState* st,
                                                            int shift, uint32_t n_tiles,
                                                            uint32_t* __restrict__ counts) {
  __shared__ uint32_t s_hist[kBins];
  const uint32_t n = st->n_valid;
  s_hist[threadIdx.x] = 0;
  __syncthreads();
  const uint32_t base = blockIdx.x * kVgTile;
  uint32_t dg[kVgRounds];
#pragma unroll
  for (int r = 0; r < kVgRounds; ++r) {
    const uint32_t i = base + r * kVgThreads + threadIdx.x;
    dg[r] = i < n ? (keys[i] >> shift) & 0xffu : 0x100u;
  }
#pragma unroll
  for (int r = 0; r < kVgRounds; ++r) {
    const uint32_t d = dg[r];
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    if (d < kBins && (peers & lanemask_lt()) == 0) atomicAdd(&s_hist[d], (uint32_t)__popc(peers));
  }
  __syncthreads();
  counts[threadIdx.x * n_tiles + blockIdx.x] = s_hist[threadIdx.x];
}

// Per digit: exclusive scan of its tile counts in place and the digit's total
// (one warp per digit; lane l holds tiles c0 + q*32 + l, so every load is one
// coalesced 128-byte row, and a warp scan per row carries the running sum).
constexpr int kScanRows = 16;

__global__ void __launch_bounds__(kVgThreads) k_radix_scan(uint32_t* __restrict__ counts, uint32_t n_tiles,
                                                           uint32_t* __restrict__ digit_total) {
  const int lane = threadIdx.x & 31;
  const uint32_t d = blockIdx.x * kVgWarps + (threadIdx.x >> 5);
  uint32_t* row = counts + (size_t)d * n_tiles;
  uint32_t carry = 0;
  for (uint32_t c0 = 0; c0 < n_tiles; c0 += 32 * kScanRows) {
    uint32_t v[kScanRows];
#pragma unroll
    for (int q = 0; q < kScanRows; ++q) {
      const uint32_t i = c0 + q * 32 + lane;
      v[q] = i < n_tiles ? row[i] : 0u;
    }
#pragma unroll
    for (int q = 0; q < kScanRows; ++q) {
      uint32_t incl = v[q];
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t a = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += a;
      }
      const uint32_t i = c0 + q * 32 + lane;
      if (i < n_tiles) row[i] = carry + incl - v[q];
      carry += __shfl_sync(0xffffffffu, incl, 31);
    }
  }
  if (lane == 0) digit_total[d] = carry;
}

// Stable scatter of one tile: items are ranked in tile order into a
// digit-sorted copy of the tile in shared memory, then written out in that
// order, so each digit's run of the tile lands in consecutive words.
__global__ void __launch_bounds__(kVgThreads) k_radix_scatter(const uint32_t* __restrict__ keys_in,
                                                              const uint32_t* __restrict__ vals_in,
                                                              uint32_t* __restrict__ keys_out,
                                                              uint32_t* __restrict__ vals_out, const VgState* st,
                                                              int shift, uint32_t n_tiles,
                                                              const uint32_t* __restrict__ offsets,
                                                              const uint32_t* __restrict__ digit_total) {
  __shared__ uint32_t s_key[kVgTile];
  __shared__ uint32_t s_val[kVgTile];
  __shared__ uint32_t s_local[kBins];  // start of each digit in the sorted tile
  __shared__ uint32_t s_run[kBins];    // next free position of each digit
  __shared__ uint32_t s_gbase[kBins];  // global position of the tile's first item of each digit
  __shared__ uint32_t s_wc[kVgWarps][kBins];
  const uint32_t n = st->n_valid;
  const uint32_t base = blockIdx.x * kVgTile;
  if (base >= n) return;
  const uint32_t tile_n = min((uint32_t)kVgTile, n - base);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t k[kVgRounds], v[kVgRounds], dg[kVgRounds];
#pragma unroll
  for (int r = 0; r < kVgRounds; ++r) {
    const uint32_t i = base + r * kVgThreads + threadIdx.x;
    const bool ok = i < n;
    k[r] = ok ? keys_in[i] : 0u;
    v[r] = ok ? vals_in[i] : 0u;
    dg[r] = ok ? (k[r] >> shift) & 0xffu : 0x100u;
  }
  s_run[threadIdx.x] = 0;
  const uint32_t tot = digit_total[threadIdx.x];
  const uint32_t goff = offsets[threadIdx.x * n_tiles + blockIdx.x];
  __syncthreads();
  // tile histogram
#pragma unroll
  for (int r = 0; r < kVgRounds; ++r) {
    const uint32_t peers = __match_any_sync(0xffffffffu, dg[r]);
    if (dg[r] < kBins && (peers & lanemask_lt()) == 0) atomicAdd(&s_run[dg[r]], (uint32_t)__popc(peers));
  }
  __syncthreads();
  // exclusive scans over the 256 digits: tile histogram and digit totals
  const uint32_t h = s_run[threadIdx.x];
  uint32_t ih = h, it = tot;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t a = __shfl_up_sync(0xffffffffu, ih, o);
    const uint32_t b = __shfl_up_sync(0xffffffffu, it, o);
    if (lane >= o) {
      ih += a;
      it += b;
    }
  }
  if (lane == 31) {
    s_wc[0][warp] = ih;
    s_wc[1][warp] = it;
  }
  __syncthreads();
  uint32_t bh = 0, bt = 0;
  for (int w = 0; w < warp; ++w) {
    bh += s_wc[0][w];
    bt += s_wc[1][w];
  }
  __syncthreads();
  s_local[threadIdx.x] = bh + ih - h;
  s_run[threadIdx.x] = bh + ih - h;
  s_gbase[threadIdx.x] = bt + it - tot + goff;
  for (int w = 0; w < kVgWarps; ++w) s_wc[w][threadIdx.x] = 0;
  __syncthreads();
  // stable ranks into the sorted tile
#pragma unroll
  for (int r = 0; r < kVgRounds; ++r) {
    const uint32_t d = dg[r];
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    const uint32_t rank = __popc(peers & lanemask_lt());
    if (d < kBins && rank == 0) s_wc[warp][d] = __popc(peers);
    __syncthreads();
    if (d < kBins) {
      uint32_t pos = s_run[d] + rank;
      for (int w = 0; w < warp; ++w) pos += s_wc[w][d];
      s_key[pos] = k[r];
      s_val[pos] = v[r];
    }
    __syncthreads();
    uint32_t t = 0;
    for (int w = 0; w < kVgWarps; ++w) {
      t += s_wc[w][threadIdx.x];
      s_wc[w][threadIdx.x] = 0;
    }
    s_run[threadIdx.x] += t;
    __syncthreads();
  }
  for (uint32_t L = threadIdx.x; L < tile_n; L += kVgThreads) {
    const uint32_t key = s_key[L];
    const uint32_t d = (key >> shift) & 0xffu;
    const uint32_t g = s_gbase[d] + (L - s_local[d]);
    keys_out[g] = key;
    vals_out[g] = s_val[L];
  }
}

// ---------------------------------------------------------------- centroids
// One warp per leaf, in batches of kBatch = 32 * kStage points.  Lane l holds
// the leaf positions base + q*32 + l (q < kStage).  A three-stage pipeline:
// the point indices of batch k+2 and the points of batch k+1 are in flight
// while lane 0 adds batch k, staged in shared memory, one point after the
// other -- the float sums run over the leaf in input order exactly as one
// thread would.  Divided by float(count) at the end.
constexpr int kStage = 8;
constexpr int kBatch = 32 * kStage;

__global__ void __launch_bounds__(kVgThreads) k_vg_centroid(const float4* __restrict__ pts,
                                                            const float* __restrict__ refl,
                                                            const float* __restrict__ amb,
                                                            const uint32_t* __restrict__ vals,
                                                            const uint32_t* __restrict__ leaf_start,
                                                            VgState* st, float4* out, float* out_refl,
                                                            float* out_amb, int direct) {
  __shared__ float4 s_p[kVgWarps][kBatch];
  __shared__ float2 s_ra[kVgWarps][kBatch];
  const uint32_t n_leaves = st->n_leaves;
  const uint32_t n_valid = st->n_valid;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint32_t warp0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t n_warps = (gridDim.x * blockDim.x) >> 5;
  const bool has_r = refl != nullptr, has_a = amb != nullptr;
  if (direct && warp0 == 0 && lane == 0) st->n_out = n_leaves;
  for (uint32_t j = warp0; j < n_leaves; j += n_warps) {
    const uint32_t b = leaf_start[j];
    const uint32_t e = j + 1 < n_leaves ? leaf_start[j + 1] : n_valid;
    uint32_t idx[kStage];   // point indices of the batch after the one in p
    float4 p[kStage];       // points of the next batch to stage
    float r[kStage], a[kStage];
#pragma unroll
    for (int q = 0; q < kStage; ++q) {
      const uint32_t k = b + q * 32 + lane;
      idx[q] = k < e ? vals[k] : 0xffffffffu;
    }
#pragma unroll
    for (int q = 0; q < kStage; ++q) {
      const uint32_t v = idx[q];
      p[q] = v != 0xffffffffu ? pts[v] : make_float4(0.f, 0.f, 0.f, 0.f);
      r[q] = has_r && v != 0xffffffffu ? refl[v] : 0.f;
      a[q] = has_a && v != 0xffffffffu ? amb[v] : 0.f;
      const uint32_t k = b + kBatch + q * 32 + lane;
      idx[q] = k < e ? vals[k] : 0xffffffffu;
    }
    float sx = 0.f, sy = 0.f, sz = 0.f, si = 0.f, sr = 0.f, sa = 0.f;
    for (uint32_t base = b; base < e; base += kBatch) {
      __syncwarp();
#pragma unroll
      for (int q = 0; q < kStage; ++q) {
        s_p[w][q * 32 + lane] = p[q];
        s_ra[w][q * 32 + lane] = make_float2(r[q], a[q]);
      }
      __syncwarp();
      // batch k+1 points, batch k+2 indices
#pragma unroll
      for (int q = 0; q < kStage; ++q) {
        const uint32_t v = idx[q];
        p[q] = v != 0xffffffffu ? pts[v] : make_float4(0.f, 0.f, 0.f, 0.f);
        r[q] = has_r && v != 0xffffffffu ? refl[v] : 0.f;
        a[q] = has_a && v != 0xffffffffu ? amb[v] : 0.f;
        const uint32_t k = base + 2 * kBatch + q * 32 + lane;
        idx[q] = k < e ? vals[k] : 0xffffffffu;
      }
      if (lane == 0) {
        const int cnt = (int)min((uint32_t)kBatch, e - base);
        for (int t = 0; t < cnt; ++t) {
          const float4 v = s_p[w][t];
          sx = __fadd_rn(sx, v.x);
          sy = __fadd_rn(sy, v.y);
          sz = __fadd_rn(sz, v.z);
          si = __fadd_rn(si, v.w);
          if (has_r || has_a) {
            const float2 ra = s_ra[w][t];
            sr = __fadd_rn(sr, ra.x);
            sa = __fadd_rn(sa, ra.y);
          }
        }
      }
    }
    if (lane == 0) {
      const float c = __uint2float_rn(e - b);
      out[j] = make_float4(__fdiv_rn(sx, c), __fdiv_rn(sy, c), __fdiv_rn(sz, c), __fdiv_rn(si, c));
      if (out_refl) out_refl[j] = __fdiv_rn(sr, c);
      if (out_amb) out_amb[j] = __fdiv_rn(sa, c);
    }
  }
}

uint32_t tiles_for(uint32_t n) { return (n + kVgTile - 1) / kVgTile; }

}  // namespace
}  // namespace phgpu

using namespace phgpu;

struct phgpu_voxel_grid {
  int device = 0;
  uint32_t max_points = 0;
  uint32_t max_tiles = 0;
  cudaStream_t st = nullptr;
  std::string err;
  float4* d_in = nullptr;
  float* d_in_refl = nullptr;
  float* d_in_amb = nullptr;
  uint32_t* keys[2] = {nullptr, nullptr};
  uint32_t* vals[2] = {nullptr, nullptr};
  uint32_t* leaf_start = nullptr;
  uint32_t* counts = nullptr;   // kBins * max_tiles
  uint32_t* offsets = nullptr;  // kBins * max_tiles
  uint32_t* digit_total = nullptr;  // kBins
  float4* d_out = nullptr;      // outputs when the caller's are host memory; per-leaf staging otherwise
  float* d_out_refl = nullptr;
  float* d_out_amb = nullptr;
  float4* d_tmp = nullptr;      // per-leaf centroids when min points > 1
  float* d_tmp_refl = nullptr;
  float* d_tmp_amb = nullptr;
  VgState* d_state = nullptr;
  VgState* h_state = nullptr;  // pinned
};

namespace {

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

thread_local std::string g_vg_create_error;

#define VG_CK(expr)                                                  \
  do {                                                               \
    cudaError_t _e = (expr);                                         \
    if (_e != cudaSuccess) {                                         \
      vg->err = std::string(#expr) + ": " + cudaGetErrorString(_e); \
      return PHGPU_ERR_CUDA;                                         \
    }                                                                \
  } while (0)

bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

}  // namespace

int phgpu_voxel_grid_create(uint32_t max_points, int32_t device, phgpu_voxel_grid** out) {
  if (!out || max_points == 0 || max_points > 0x7fffffffu) {
    g_vg_create_error = "max_points must be in [1, 2^31)";
    return PHGPU_ERR_INVALID;
  }
  *out = nullptr;
  int n_dev = 0;
  if (cudaGetDeviceCount(&n_dev) != cudaSuccess || device < 0 || device >= n_dev) {
    g_vg_create_error = "no such CUDA device";
    return PHGPU_ERR_CUDA;
  }
  DeviceGuard g(device);
  phgpu_voxel_grid* vg = new phgpu_voxel_grid();
  vg->device = device;
  vg->max_points = max_points;
  vg->max_tiles = tiles_for(max_points);
  const size_t P = max_points;
  const size_t words = (size_t)kBins * vg->max_tiles;
  cudaError_t e = cudaStreamCreateWithFlags(&vg->st, cudaStreamNonBlocking);
  auto alloc = [&](void** p, size_t bytes) {
    if (e == cudaSuccess) e = cudaMalloc(p, bytes);
  };
  alloc((void**)&vg->d_in, P * sizeof(float4));
  alloc((void**)&vg->d_in_refl, P * sizeof(float));
  alloc((void**)&vg->d_in_amb, P * sizeof(float));
  for (int k = 0; k < 2; ++k) {
    alloc((void**)&vg->keys[k], P * sizeof(uint32_t));
    alloc((void**)&vg->vals[k], P * sizeof(uint32_t));
  }
  alloc((void**)&vg->leaf_start, P * sizeof(uint32_t));
  alloc((void**)&vg->counts, words * sizeof(uint32_t));
  alloc((void**)&vg->offsets, words * sizeof(uint32_t));
  alloc((void**)&vg->digit_total, kBins * sizeof(uint32_t));
  alloc((void**)&vg->d_out, P * sizeof(float4));
  alloc((void**)&vg->d_out_refl, P * sizeof(float));
  alloc((void**)&vg->d_out_amb, P * sizeof(float));
  alloc((void**)&vg->d_tmp, P * sizeof(float4));
  alloc((void**)&vg->d_tmp_refl, P * sizeof(float));
  alloc((void**)&vg->d_tmp_amb, P * sizeof(float));
  alloc((void**)&vg->d_state, sizeof(VgState));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&vg->h_state, sizeof(VgState));
  if (e != cudaSuccess) {
    g_vg_create_error = std::string("voxel grid allocation: ") + cudaGetErrorString(e);
    phgpu_voxel_grid_destroy(vg);
    return e == cudaErrorMemoryAllocation ? PHGPU_ERR_MEMORY : PHGPU_ERR_CUDA;
  }
  *out = vg;
  return PHGPU_OK;
}

int phgpu_voxel_grid_destroy(phgpu_voxel_grid* vg) {
  if (!vg) return PHGPU_ERR_INVALID;
  DeviceGuard g(vg->device);
  if (vg->st) cudaStreamSynchronize(vg->st);
  void* bufs[] = {vg->d_in, vg->d_in_refl, vg->d_in_amb, vg->keys[0], vg->keys[1], vg->vals[0], vg->vals[1],
                  vg->leaf_start, vg->counts, vg->offsets, vg->digit_total, vg->d_out, vg->d_out_refl, vg->d_out_amb, vg->d_tmp,
                  vg->d_tmp_refl, vg->d_tmp_amb, vg->d_state};
  for (void* b : bufs)
    if (b) cudaFree(b);
  if (vg->h_state) cudaFreeHost(vg->h_state);
  if (vg->st) cudaStreamDestroy(vg->st);
  delete vg;
  return PHGPU_OK;
}

const char* phgpu_voxel_grid_last_error(const phgpu_voxel_grid* vg) {
  return vg ? vg->err.c_str() : g_vg_create_error.c_str();
}

int phgpu_voxel_grid_filter(phgpu_voxel_grid* vg, const phgpu_cloud* in, const float leaf[3],
                            uint32_t min_points_per_voxel, float* out_xyzi, float* out_reflectivity,
                            float* out_ambient, int out_on_device, uint32_t* n_out) {
  if (!vg) return PHGPU_ERR_INVALID;
  vg->err.clear();
  if (!in || !leaf || !out_xyzi || !n_out) {
    vg->err = "null argument";
    return PHGPU_ERR_INVALID;
  }
  if (in->n_points > vg->max_points) {
    vg->err = "cloud larger than max_points";
    return PHGPU_ERR_INVALID;
  }
  for (int a = 0; a < 3; ++a)
    if (!(leaf[a] > 0.f) || !isfinite(leaf[a])) {
      vg->err = "leaf sizes must be positive and finite";
      return PHGPU_ERR_INVALID;
    }
  if ((in->on_device && in->n_points && !aligned16(in->xyzi)) || (out_on_device && !aligned16(out_xyzi))) {
    vg->err = "device xyzi buffers must be 16-byte aligned";
    return PHGPU_ERR_INVALID;
  }
  DeviceGuard g(vg->device);
  cudaStream_t st = vg->st;
  const uint32_t n = in->n_points;
  *n_out = 0;
  if (n == 0) return PHGPU_OK;

  const float4* pts = (const float4*)in->xyzi;
  const float* refl = in->reflectivity;
  const float* amb = in->ambient;
  if (!in->on_device) {
    VG_CK(cudaMemcpyAsync(vg->d_in, in->xyzi, (size_t)n * sizeof(float4), cudaMemcpyHostToDevice, st));
    pts = vg->d_in;
    if (refl) {
      VG_CK(cudaMemcpyAsync(vg->d_in_refl, refl, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, st));
      refl = vg->d_in_refl;
    }
    if (amb) {
      VG_CK(cudaMemcpyAsync(vg->d_in_amb, amb, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, st));
      amb = vg->d_in_amb;
    }
  }
  // outputs: the caller's device buffers, or device staging for host ones
  float4* out = out_on_device ? (float4*)out_xyzi : vg->d_out;
  float* o_refl = refl && out_reflectivity ? (out_on_device ? out_reflectivity : vg->d_out_refl) : nullptr;
  float* o_amb = amb && out_ambient ? (out_on_device ? out_ambient : vg->d_out_amb) : nullptr;

  const float inv[3] = {1.0f / leaf[0], 1.0f / leaf[1], 1.0f / leaf[2]};
  const uint32_t tiles = tiles_for(n);
  VgState* s = vg->d_state;
  int launches = 0;
  VG_CK(cudaMemsetAsync(s, 0, sizeof(VgState), st));
  const int bounds_blocks = (int)std::min<uint32_t>((n + kVgThreads - 1) / kVgThreads, (uint32_t)kBoundsBlocks);
  k_vg_bounds<<<bounds_blocks, kVgThreads, 0, st>>>(pts, n, vg->offsets);
  k_vg_plan<<<1, 32, 0, st>>>(vg->offsets, bounds_blocks, s, inv[0], inv[1], inv[2]);
  launches += 2;

  ValidOp vop{pts, n, {inv[0], inv[1], inv[2]}, s, vg->keys[0], vg->vals[0]};
  k_flag_count<ValidOp><<<tiles, kVgThreads, 0, st>>>(vop, vg->counts);
  k_scan_words<<<1, kScanThreads, 0, st>>>(vg->counts, tiles, vg->offsets, &s->n_valid);
  k_flag_scatter<ValidOp><<<tiles, kVgThreads, 0, st>>>(vop, vg->offsets);
  launches += 3;

  int cur = 0;
  for (int pass = 0; pass < 4; ++pass) {
    const int shift = 8 * pass;
    k_radix_count<<<tiles, kVgThreads, 0, st>>>(vg->keys[cur], s, shift, tiles, vg->counts);
    k_radix_scan<<<kBins / kVgWarps, kVgThreads, 0, st>>>(vg->counts, tiles, vg->digit_total);
    k_radix_scatter<<<tiles, kVgThreads, 0, st>>>(vg->keys[cur], vg->vals[cur], vg->keys[cur ^ 1],
                                                  vg->vals[cur ^ 1], s, shift, tiles, vg->counts,
                                                  vg->digit_total);
    cur ^= 1;
    launches += 3;
  }

  HeadOp hop{vg->keys[cur], s, vg->leaf_start};
  k_flag_count<HeadOp><<<tiles, kVgThreads, 0, st>>>(hop, vg->counts);
  k_scan_words<<<1, kScanThreads, 0, st>>>(vg->counts, tiles, vg->offsets, &s->n_leaves);
  k_flag_scatter<HeadOp><<<tiles, kVgThreads, 0, st>>>(hop, vg->offsets);
  launches += 3;

  const bool direct = min_points_per_voxel <= 1;
  const uint32_t leaf_blocks = std::min<uint32_t>((n + kVgWarps - 1) / kVgWarps, 148u * 16u);
  k_vg_centroid<<<leaf_blocks, kVgThreads, 0, st>>>(pts, o_refl ? refl : nullptr, o_amb ? amb : nullptr,
                                                    vg->vals[cur], vg->leaf_start, s, direct ? out : vg->d_tmp,
                                                    direct ? o_refl : (o_refl ? vg->d_tmp_refl : nullptr),
                                                    direct ? o_amb : (o_amb ? vg->d_tmp_amb : nullptr), direct ? 1 : 0);
  launches += 1;
  if (!direct) {
    KeepOp kop{vg->leaf_start, s, min_points_per_voxel, vg->d_tmp, vg->d_tmp_refl, vg->d_tmp_amb, out, o_refl, o_amb};
    k_flag_count<KeepOp><<<tiles, kVgThreads, 0, st>>>(kop, vg->counts);
    k_scan_words<<<1, kScanThreads, 0, st>>>(vg->counts, tiles, vg->offsets, &s->n_out);
    k_flag_scatter<KeepOp><<<tiles, kVgThreads, 0, st>>>(kop, vg->offsets);
    launches += 3;
  }
  count_launches(launches);
  VG_CK(cudaGetLastError());
  VG_CK(cudaMemcpyAsync(vg->h_state, s, sizeof(VgState), cudaMemcpyDeviceToHost, st));
  VG_CK(cudaStreamSynchronize(st));
  const VgState& hs = *vg->h_state;
  if (hs.status == kVgRange) {
    vg->err = "leaf indices leave the int32 / 32-bit cell range for this leaf size";
    return PHGPU_ERR_LIMIT;
  }
  const cudaMemcpyKind to_out = out_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  if (hs.status == kVgOverflow) {
    // the reference's "Integer indices would overflow" branch: output = input
    VG_CK(cudaMemcpyAsync(out_xyzi, pts, (size_t)n * sizeof(float4), to_out, st));
    if (o_refl) VG_CK(cudaMemcpyAsync(out_reflectivity, refl, (size_t)n * sizeof(float), to_out, st));
    if (o_amb) VG_CK(cudaMemcpyAsync(out_ambient, amb, (size_t)n * sizeof(float), to_out, st));
    VG_CK(cudaStreamSynchronize(st));
    *n_out = n;
    return PHGPU_OK;
  }
  const uint32_t m = hs.status == kVgOk ? hs.n_out : 0u;
  if (!out_on_device && m) {
    VG_CK(cudaMemcpyAsync(out_xyzi, out, (size_t)m * sizeof(float4), cudaMemcpyDeviceToHost, st));
    if (o_refl) VG_CK(cudaMemcpyAsync(out_reflectivity, o_refl, (size_t)m * sizeof(float), cudaMemcpyDeviceToHost, st));
    if (o_amb) VG_CK(cudaMemcpyAsync(out_ambient, o_amb, (size_t)m * sizeof(float), cudaMemcpyDeviceToHost, st));
    VG_CK(cudaStreamSynchronize(st));
  }
  *n_out = m;
  return PHGPU_OK;
}
