// Shared device helpers for the PHASER registration kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

namespace phgpu {

constexpr int kMaxLevels = 8;

// Positional Laplace-pyramid fusion rule on an FFT-shifted linear index
// (phaser_core/src/backend/fusion/laplace-pyramid.cc:60-104 with
// pyramid-struct.cc:17-29).  For each level: [lb, eub) recurses into the next
// level, [eub, sub) is the zero slot left by the PyramidStruct / expand()
// rounding mismatch, everything else takes the max-energy channel; after the
// last level the channel mean.  Band tables are computed on the host with the
// reference's float arithmetic.
struct FusionBands {
  int levels;
  uint32_t n;
  uint32_t lb[kMaxLevels];
  uint32_t eub[kMaxLevels];
  uint32_t sub[kMaxLevels];
};

enum FusionOp : int { kFuseMax = 0, kFuseZero = 1, kFuseMean = 2 };

__host__ __device__ inline int fusion_op(uint32_t p, const FusionBands& b) {
  for (int l = 0; l < b.levels; ++l) {
    if (p >= b.lb[l] && p < b.eub[l]) {
      p -= b.lb[l];
      continue;
    }
    if (p >= b.lb[l] && p < b.sub[l]) return kFuseZero;
    return kFuseMax;
  }
  return kFuseMean;
}

// Order-preserving packing for a first-occurrence argmax with atomicMax:
// larger value wins, equal values -> smaller index wins.
__device__ __forceinline__ uint32_t float_order_bits(float v) {
  const uint32_t u = __float_as_uint(v);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__host__ __device__ inline float float_from_order_bits(uint32_t o) {
  const uint32_t u = (o & 0x80000000u) ? (o & 0x7fffffffu) : ~o;
#ifdef __CUDA_ARCH__
  return __uint_as_float(u);
#else
  float f;
  memcpy(&f, &u, 4);
  return f;
#endif
}
__device__ __forceinline__ unsigned long long pack_argmax(float v, uint32_t idx) {
  return ((unsigned long long)float_order_bits(v) << 32) | (unsigned long long)(0xffffffffu - idx);
}
__host__ __device__ inline uint32_t unpack_index(unsigned long long k) {
  return 0xffffffffu - (uint32_t)(k & 0xffffffffull);
}

// Warp-level reduction of a packed argmax key followed by one atomicMax per
// warp (1-D blocks).  The last warp of a block whose size is not a multiple
// of 32 (1000 threads at N = 200) has lanes that do not exist, and a shuffle
// from such a lane returns an undefined value: its lanes commit one by one.
__device__ __forceinline__ void warp_argmax_commit(unsigned long long key, unsigned long long* dst) {
  if ((threadIdx.x | 31u) >= blockDim.x) {
    if (key) atomicMax(dst, key);
    return;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long other = __shfl_xor_sync(0xffffffffu, key, o);
    key = other > key ? other : key;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(dst, key);
}

// Complex sums as packed FP32 pairs (one FADD2 / FFMA2 for both components).
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }

}  // namespace phgpu
