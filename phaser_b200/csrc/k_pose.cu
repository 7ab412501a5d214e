// Rotation pose of the SO(3) argmax on the device, so a registration is one
// asynchronous chain: rotation argmax -> pose -> transform of the source cloud
// -> translation, without a host round trip in between.
//
// Reference behaviour (phaser_common/src/common/rotation-utils.cc):
// convertSO3toZYZ (197-208), ConvertZYZtoQuaternion (101-107),
// ConvertQuaternionToXYZ / fromRotation (86-93, 190-196) and RotateAroundXYZ
// (17-24, 109-143).  Every operation is written out in the order of the host
// restatement (capi.cu, phgpu_pose_from_bin) with explicit IEEE roundings, so
// nothing is contracted differently; the double trig functions are CUDA's
// and glibc's on the two sides, so the host compares the device transform
// with its own after the registration and redoes the translation on the rare
// difference.  float cos / sin are correctly rounded on both sides.
#include <math.h>

#include "kernels.h"

namespace phgpu {

__device__ __forceinline__ void dquat_product(const double* a, const double* b, double* r) {
  r[0] = __dsub_rn(__dsub_rn(__dsub_rn(__dmul_rn(a[0], b[0]), __dmul_rn(a[1], b[1])), __dmul_rn(a[2], b[2])),
                   __dmul_rn(a[3], b[3]));
  r[1] = __dsub_rn(__dadd_rn(__dadd_rn(__dmul_rn(a[0], b[1]), __dmul_rn(a[1], b[0])), __dmul_rn(a[2], b[3])),
                   __dmul_rn(a[3], b[2]));
  r[2] = __dsub_rn(__dadd_rn(__dadd_rn(__dmul_rn(a[0], b[2]), __dmul_rn(a[2], b[0])), __dmul_rn(a[3], b[1])),
                   __dmul_rn(a[1], b[3]));
  r[3] = __dsub_rn(__dadd_rn(__dadd_rn(__dmul_rn(a[0], b[3]), __dmul_rn(a[3], b[0])), __dmul_rn(a[1], b[2])),
                   __dmul_rn(a[2], b[1]));
}

__device__ void device_pose(uint32_t loc, uint32_t bw, float* T12) {
  // convertSO3toZYZ
  const double dbw = (double)bw;
  const double q4 = __dmul_rn(__dmul_rn(4.0, dbw), dbw);
  const int32_t ii = (int32_t)floor(__ddiv_rn((double)loc, q4));
  const int32_t tmp = (int32_t)__dsub_rn((double)loc, __dmul_rn(__dmul_rn(__dmul_rn((double)ii, 4.0), dbw), dbw));
  const int32_t jj = (int32_t)floor(__ddiv_rn((double)tmp, __dmul_rn(2.0, dbw)));
  const int32_t kk = (int32_t)loc - (ii * 4 * (int32_t)bw * (int32_t)bw) - jj * (2 * (int32_t)bw);
  double z[3];
  z[0] = __ddiv_rn(__dmul_rn(M_PI, (double)jj), dbw);
  z[1] = __ddiv_rn(__dmul_rn(M_PI, (double)(2 * ii + 1)), __dmul_rn(4.0, dbw));
  z[2] = __ddiv_rn(__dmul_rn(M_PI, (double)kk), dbw);
  // ConvertZYZtoQuaternion: AngleAxis(a, Z) * AngleAxis(b, Y) * AngleAxis(c, Z)
  const double qa[4] = {cos(0.5 * z[0]), 0.0, 0.0, sin(0.5 * z[0])};
  const double qb[4] = {cos(0.5 * z[1]), 0.0, sin(0.5 * z[1]), 0.0};
  const double qc[4] = {cos(0.5 * z[2]), 0.0, 0.0, sin(0.5 * z[2])};
  double t[4], q[4];
  dquat_product(qa, qb, t);
  dquat_product(t, qc, q);
  // ConvertQuaternionToXYZ
  const double qw = q[0], qx = q[1], qy = q[2], qz = q[3];
  const double r11 = __dmul_rn(-2.0, __dsub_rn(__dmul_rn(qy, qz), __dmul_rn(qw, qx)));
  const double r12 =
      __dadd_rn(__dsub_rn(__dsub_rn(__dmul_rn(qw, qw), __dmul_rn(qx, qx)), __dmul_rn(qy, qy)), __dmul_rn(qz, qz));
  const double r21 = __dmul_rn(2.0, __dadd_rn(__dmul_rn(qx, qz), __dmul_rn(qw, qy)));
  const double r31 = __dmul_rn(-2.0, __dsub_rn(__dmul_rn(qx, qy), __dmul_rn(qw, qz)));
  const double r32 =
      __dsub_rn(__dsub_rn(__dadd_rn(__dmul_rn(qw, qw), __dmul_rn(qx, qx)), __dmul_rn(qy, qy)), __dmul_rn(qz, qz));
  const double e2 = -atan2(r31, r32);
  const double e1 = asin(r21);
  const double e0 = atan2(r11, r12);
  // RotateAroundXYZ: Rx(a) * Ry(b) * Rz(c) in float
  const float a = (float)e0, b = (float)e1, c = (float)e2;
  const float ca = (float)cos((double)a), sa = (float)sin((double)a);
  const float cb = (float)cos((double)b), sb = (float)sin((double)b);
  const float cc = (float)cos((double)c), sc = (float)sin((double)c);
  const float X[3][3] = {{1.f, 0.f, 0.f}, {0.f, ca, -sa}, {0.f, sa, ca}};
  const float Y[3][3] = {{cb, 0.f, sb}, {0.f, 1.f, 0.f}, {-sb, 0.f, cb}};
  const float Z[3][3] = {{cc, sc, 0.f}, {-sc, cc, 0.f}, {0.f, 0.f, 1.f}};
  float XY[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      float s = 0.0f;
      for (int k = 0; k < 3; ++k) s = __fadd_rn(s, __fmul_rn(X[i][k], Y[k][j]));
      XY[i][j] = s;
    }
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) {
      float s = 0.0f;
      for (int k = 0; k < 3; ++k) s = __fadd_rn(s, __fmul_rn(XY[i][k], Z[k][j]));
      T12[4 * i + j] = s;
    }
    T12[4 * i + 3] = 0.0f;
  }
}

__global__ void k_pose(PoseBatch b) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= b.count) return;
  const uint32_t bin = unpack_index(*b.argmax[r]);
  device_pose(bin, b.bw_out, b.T[r]);
}

cudaError_t launch_pose(const PoseBatch& b, cudaStream_t st) {
  if (b.count < 1 || b.count > kMaxWave) return cudaErrorInvalidValue;
  k_pose<<<1, 32, 0, st>>>(b);
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace phgpu
