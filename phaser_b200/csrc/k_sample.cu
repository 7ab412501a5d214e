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
// cells), with exact per-cell bounding boxes.  A query first takes an upper
// bound from one representative point per non-empty coarse cell, then scans
// only cells whose box lies within that bound (with a 1e-5 relative margin so
// float rounding can never prune the true nearest point).
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

__global__ void k_project(const float4* __restrict__ xyzi, int P, float4* __restrict__ proj,
                          double* __restrict__ range, uint32_t* __restrict__ key,
                          uint32_t* __restrict__ cell_count) {
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
  const uint32_t k = cell_key(ox, oy, oz);
  key[i] = k;
  atomicAdd(&cell_count[k], 1u);
}

// Exclusive scan of the 32768 fine-cell counts (one block of 1024 threads).
__global__ void k_cell_scan(const uint32_t* __restrict__ count, uint32_t* __restrict__ start) {
  __shared__ uint32_t part[1024];
  const int t = threadIdx.x;
  constexpr int per = kFineCells / 1024;
  uint32_t local[per];
  uint32_t s = 0;
#pragma unroll
  for (int j = 0; j < per; ++j) {
    local[j] = count[t * per + j];
    s += local[j];
  }
  part[t] = s;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    const uint32_t v = t >= off ? part[t - off] : 0u;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  uint32_t run = part[t] - s;
#pragma unroll
  for (int j = 0; j < per; ++j) {
    start[t * per + j] = run;
    run += local[j];
  }
  if (t == 1023) start[kFineCells] = part[1023];
}

__global__ void k_scatter(int P, const float4* __restrict__ proj, const uint32_t* __restrict__ key,
                          const uint32_t* __restrict__ start, uint32_t* __restrict__ cursor,
                          float4* __restrict__ sorted) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P) return;
  const uint32_t k = key[i];
  const uint32_t slot = start[k] + atomicAdd(&cursor[k], 1u);
  const float4 p = proj[i];
  sorted[slot] = make_float4(p.x, p.y, p.z, __int_as_float(i));
}

__global__ void k_fine_bounds(const float4* __restrict__ sorted, const uint32_t* __restrict__ start,
                              float* __restrict__ fbox) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= kFineCells) return;
  const uint32_t s = start[c], e = start[c + 1];
  float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint32_t j = s; j < e; ++j) {
    const float4 p = sorted[j];
    lo[0] = fminf(lo[0], p.x);
    lo[1] = fminf(lo[1], p.y);
    lo[2] = fminf(lo[2], p.z);
    hi[0] = fmaxf(hi[0], p.x);
    hi[1] = fmaxf(hi[1], p.y);
    hi[2] = fmaxf(hi[2], p.z);
  }
  float* b = fbox + 6 * c;
  b[0] = lo[0];
  b[1] = lo[1];
  b[2] = lo[2];
  b[3] = hi[0];
  b[4] = hi[1];
  b[5] = hi[2];
}

// Coarse cells: merged boxes and the compact list of non-empty cells.
// clist entries: {start, count, coarse id, pad} + box (6 floats).
__global__ void k_coarse_bounds(const uint32_t* __restrict__ start, const float* __restrict__ fbox,
                                uint4* __restrict__ clist, float* __restrict__ cbox,
                                uint32_t* __restrict__ n_coarse) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= kCoarseCells) return;
  const uint32_t s = start[c * 64], e = start[c * 64 + 64];
  if (e == s) return;
  float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int f = 0; f < 64; ++f) {
    const int fc = c * 64 + f;
    if (start[fc + 1] == start[fc]) continue;
    const float* b = fbox + 6 * fc;
    for (int a = 0; a < 3; ++a) {
      lo[a] = fminf(lo[a], b[a]);
      hi[a] = fmaxf(hi[a], b[3 + a]);
    }
  }
  const uint32_t slot = atomicAdd(n_coarse, 1u);
  clist[slot] = make_uint4(s, e - s, (uint32_t)c, 0u);
  float* o = cbox + 6 * slot;
  for (int a = 0; a < 3; ++a) {
    o[a] = lo[a];
    o[3 + a] = hi[a];
  }
}

__device__ __forceinline__ float box_lb2(float qx, float qy, float qz, const float* b) {
  const float dx = fmaxf(fmaxf(b[0] - qx, qx - b[3]), 0.0f);
  const float dy = fmaxf(fmaxf(b[1] - qy, qy - b[4]), 0.0f);
  const float dz = fmaxf(fmaxf(b[2] - qz, qz - b[5]), 0.0f);
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

constexpr int kQueryThreads = 256;

// One thread per grid direction.  Writes the sampled channels
// {range, intensity, reflectivity, ambient} (float) into out[ch][query] for
// ch < n_out_ch and the nearest index (or -1) into nn_idx.
__global__ void __launch_bounds__(kQueryThreads)
k_nn_query(int nq, const float4* __restrict__ grid, const float4* __restrict__ sorted,
           const uint32_t* __restrict__ fstart, const float* __restrict__ fbox,
           const uint4* __restrict__ clist, const float* __restrict__ cbox,
           const uint32_t* __restrict__ n_coarse_p, float max_sq, const float4* __restrict__ xyzi,
           const double* __restrict__ range, const float* __restrict__ refl,
           const float* __restrict__ amb, int n_out_ch, float* __restrict__ out,
           int32_t* __restrict__ nn_idx) {
  __shared__ uint4 s_list[kCoarseCells];
  __shared__ float s_box[kCoarseCells * 6];
  __shared__ float4 s_rep[kCoarseCells];
  const int nc = (int)*n_coarse_p;
  for (int i = threadIdx.x; i < nc; i += blockDim.x) {
    const uint4 e = clist[i];
    s_list[i] = e;
    s_rep[i] = sorted[e.x];
  }
  for (int i = threadIdx.x; i < nc * 6; i += blockDim.x) s_box[i] = cbox[i];
  __syncthreads();
  const int qi = blockIdx.x * blockDim.x + threadIdx.x;
  if (qi >= nq) return;
  const float4 q = grid[qi];
  float best = INFINITY;
  int bidx = 0x7fffffff;
  for (int c = 0; c < nc; ++c) {
    const float4 r = s_rep[c];
    nn_update(ref_dist2(q.x, q.y, q.z, r), __float_as_int(r.w), best, bidx);
  }
  for (int c = 0; c < nc; ++c) {
    if (box_lb2(q.x, q.y, q.z, s_box + 6 * c) * 0.99999f > best) continue;
    const uint32_t cid = s_list[c].z;
    for (int f = 0; f < 64; ++f) {
      const int fc = (int)cid * 64 + f;
      const uint32_t s = __ldg(&fstart[fc]), e = __ldg(&fstart[fc + 1]);
      if (s == e) continue;
      if (box_lb2(q.x, q.y, q.z, fbox + 6 * fc) * 0.99999f > best) continue;
      for (uint32_t j = s; j < e; ++j) {
        const float4 p = sorted[j];
        nn_update(ref_dist2(q.x, q.y, q.z, p), __float_as_int(p.w), best, bidx);
      }
    }
  }
  const bool ok = (bidx != 0x7fffffff) && !(best > max_sq);
  float v[4] = {0.f, 0.f, 0.f, 0.f};
  if (ok) {
    v[0] = (float)range[bidx];
    v[1] = xyzi[bidx].w;
    v[2] = refl ? refl[bidx] : 0.0f;
    v[3] = amb ? amb[bidx] : 0.0f;
  }
  for (int ch = 0; ch < n_out_ch; ++ch) out[(size_t)ch * nq + qi] = v[ch];
  if (nn_idx) nn_idx[qi] = ok ? bidx : -1;
}

// ---------------------------------------------------------------- launcher

size_t sampler_scratch_bytes(int max_points) {
  size_t b = 0;
  b += (size_t)max_points * sizeof(float4);   // proj
  b += (size_t)max_points * sizeof(double);   // range
  b += (size_t)max_points * sizeof(uint32_t); // key
  b += (size_t)max_points * sizeof(float4);   // sorted
  b += (size_t)kFineCells * sizeof(uint32_t) * 2;  // count, cursor
  b += (size_t)(kFineCells + 1) * sizeof(uint32_t);
  b += (size_t)kFineCells * 6 * sizeof(float);
  b += (size_t)kCoarseCells * sizeof(uint4);
  b += (size_t)kCoarseCells * 6 * sizeof(float);
  b += 256;
  return b + 16 * 256;
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
  uint32_t* start = (uint32_t*)carve(p, (size_t)(kFineCells + 1) * sizeof(uint32_t));
  float* fbox = (float*)carve(p, (size_t)kFineCells * 6 * sizeof(float));
  uint4* clist = (uint4*)carve(p, (size_t)kCoarseCells * sizeof(uint4));
  float* cbox = (float*)carve(p, (size_t)kCoarseCells * 6 * sizeof(float));
  uint32_t* ncoarse = (uint32_t*)carve(p, 256);

  cudaMemsetAsync(count, 0, (size_t)kFineCells * sizeof(uint32_t), st);
  cudaMemsetAsync(cursor, 0, (size_t)kFineCells * sizeof(uint32_t), st);
  cudaMemsetAsync(ncoarse, 0, sizeof(uint32_t), st);
  const int P = a.n_points;
  if (P > 0) {
    k_project<<<(P + 255) / 256, 256, 0, st>>>(a.xyzi, P, proj, range, key, count);
  }
  k_cell_scan<<<1, 1024, 0, st>>>(count, start);
  if (P > 0) {
    k_scatter<<<(P + 255) / 256, 256, 0, st>>>(P, proj, key, start, cursor, sorted);
  }
  k_fine_bounds<<<kFineCells / 256, 256, 0, st>>>(sorted, start, fbox);
  k_coarse_bounds<<<kCoarseCells / 128, 128, 0, st>>>(start, fbox, clist, cbox, ncoarse);
  k_nn_query<<<(a.n_queries + kQueryThreads - 1) / kQueryThreads, kQueryThreads, 0, st>>>(
      a.n_queries, a.grid, sorted, start, fbox, clist, cbox, ncoarse, a.max_sq, a.xyzi, range,
      a.refl, a.amb, a.n_out_ch, a.out, a.nn_idx);
  return cudaGetLastError();
}

}  // namespace phgpu
