// Host side of the C ABI (include/phaser_gpu.h): per-configuration context,
// FFT plans, fusion band tables, the reference's host pose arithmetic and the
// plain one-pair-at-a-time pipeline.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/phaser_gpu.h"
#include "ctx.h"
#include "kernels.h"

using namespace phgpu;

static thread_local std::string g_create_error;

#define CK(expr)                                                                   \
  do {                                                                             \
    cudaError_t _e = (expr);                                                       \
    if (_e != cudaSuccess) {                                                       \
      ctx->err = std::string(#expr) + ": " + cudaGetErrorString(_e);               \
      return PHGPU_ERR_CUDA;                                                       \
    }                                                                              \
  } while (0)

#define CKC(c, expr)                                                               \
  do {                                                                             \
    cudaError_t _e = (expr);                                                       \
    if (_e != cudaSuccess) {                                                       \
      (c)->err = std::string(#expr) + ": " + cudaGetErrorString(_e);               \
      return PHGPU_ERR_CUDA;                                                       \
    }                                                                              \
  } while (0)

#define CKV(expr)                                                                  \
  do {                                                                             \
    int _r = (expr);                                                               \
    if (_r != PHGPU_OK) return _r;                                                 \
  } while (0)

// ------------------------------------------------------------------ helpers

namespace phgpu {

// Radix preference orders of runtime FFT plans (a tuned parameter): radix 8
// first; radix 4 first; odd radices first.
static const int kRadixOrders[3][8] = {{8, 4, 2, 5, 3, 7, 11, 13}, {4, 2, 8, 5, 3, 7, 11, 13},
                                       {5, 3, 7, 11, 13, 8, 4, 2}};

// Stages of a runtime plan of length n in radix order `order`; false when n
// has a prime factor above the generic radix limit.
bool fft_plan_radices(int n, int order, FftPlan* p) {
  const int* pref = kRadixOrders[(order >= 0 && order < 3) ? order : 0];
  int m = n, ns = 0;
  for (int i = 0; i < 8; ++i) {
    const int r = pref[i];
    while (m % r == 0 && ns < kMaxFftStages) {
      p->radix[ns++] = r;
      m /= r;
    }
  }
  for (int r = 17; m > 1 && r <= kMaxGenericRadix && ns < kMaxFftStages; r += 2) {
    while (m % r == 0 && ns < kMaxFftStages) {
      p->radix[ns++] = r;
      m /= r;
    }
  }
  if (m != 1 || n < 1) return false;
  p->n = n;
  p->nstage = ns;
  int L = n;
  for (int s = 0; s < ns; ++s) {
    p->L[s] = L;
    L /= p->radix[s];
  }
  return true;
}

bool make_fft_plan(int n, FftPlan* p, float2** d_tw, std::string* err) {
  memset(p, 0, sizeof(*p));
  if (!fft_plan_radices(n, 0, p)) {
    *err = "FFT length " + std::to_string(n) + " has a prime factor above " +
           std::to_string(kMaxGenericRadix) + " (unsupported)";
    return false;
  }
  std::vector<float2> tw(n);
  for (int t = 0; t < n; ++t) {
    const double a = -2.0 * M_PI * (double)t / (double)n;
    tw[t] = make_float2((float)cos(a), (float)sin(a));
  }
  if (cudaMalloc(d_tw, sizeof(float2) * n) != cudaSuccess) {
    *err = "cudaMalloc twiddles failed";
    return false;
  }
  cudaMemcpy(*d_tw, tw.data(), sizeof(float2) * n, cudaMemcpyHostToDevice);
  p->tw = *d_tw;
  return true;
}

// PyramidStruct (pyramid-struct.cc:17-29) and LaplacePyramid::expand
// (laplace-pyramid.cc:40-58) bounds with the reference's float arithmetic.
FusionBands make_bands(uint32_t n, int levels, float div) {
  FusionBands b;
  memset(&b, 0, sizeof(b));
  b.levels = levels;
  b.n = n;
  uint32_t cur = n;
  for (int l = 0; l < levels; ++l) {
    const float lower = (float)cur / div;
    const uint32_t upper = (uint32_t)roundf((float)cur - lower);
    const uint32_t lb = (uint32_t)roundf(lower);
    const uint32_t elb = (uint32_t)roundf((float)cur / div);
    b.lb[l] = lb;
    b.sub[l] = upper;
    b.eub[l] = cur - elb;
    cur = upper - lb;
  }
  return b;
}

}  // namespace phgpu

// RotationUtils::convertSO3toZYZ (rotation-utils.cc:197-208).
static void bin_to_zyz(uint32_t loc, uint32_t bw, double* zyz) {
  const int32_t ii = (int32_t)floor(loc / (4. * bw * bw));
  const int32_t tmp = (int32_t)(loc - (ii * 4. * bw * bw));
  const int32_t jj = (int32_t)floor(tmp / (2. * bw));
  const int32_t kk = (int32_t)loc - (ii * 4 * (int32_t)bw * (int32_t)bw) - jj * (2 * (int32_t)bw);
  const double b = (double)bw;
  zyz[0] = M_PI * jj / b;
  zyz[1] = M_PI * (2 * ii + 1) / (4. * bw);
  zyz[2] = M_PI * kk / b;
}

// Hamilton product in the term order of Eigen's generic quat_product.
static void quat_product(const double* a, const double* b, double* r) {
  r[0] = a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3];
  r[1] = a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2];
  r[2] = a[0] * b[2] + a[2] * b[0] + a[3] * b[1] - a[1] * b[3];
  r[3] = a[0] * b[3] + a[3] * b[0] + a[1] * b[2] - a[2] * b[1];
}

// ConvertZYZtoQuaternion: AngleAxis(a, Z) * AngleAxis(b, Y) * AngleAxis(c, Z)
// (rotation-utils.cc:101-107).
static void zyz_to_quat(const double* z, double* q) {
  const double qa[4] = {cos(0.5 * z[0]), 0.0, 0.0, sin(0.5 * z[0])};
  const double qb[4] = {cos(0.5 * z[1]), 0.0, sin(0.5 * z[1]), 0.0};
  const double qc[4] = {cos(0.5 * z[2]), 0.0, 0.0, sin(0.5 * z[2])};
  double t[4];
  quat_product(qa, qb, t);
  quat_product(t, qc, q);
}

// ConvertQuaternionToXYZ / fromRotation (rotation-utils.cc:86-93, 190-196).
static void quat_to_xyz(const double* q, double* e) {
  const double qw = q[0], qx = q[1], qy = q[2], qz = q[3];
  const double r11 = -2 * (qy * qz - qw * qx);
  const double r12 = qw * qw - qx * qx - qy * qy + qz * qz;
  const double r21 = 2 * (qx * qz + qw * qy);
  const double r31 = -2 * (qx * qy - qw * qz);
  const double r32 = qw * qw + qx * qx - qy * qy - qz * qz;
  e[2] = -atan2(r31, r32);
  e[1] = asin(r21);
  e[0] = atan2(r11, r12);
}

static void xyz_to_transform(const double* e, float* T12);

int phgpu_pose_from_bin(uint32_t bin, uint32_t bw_out, double* zyz, double* quat, double* xyz, float* T12) {
  double z[3], q[4], e[3];
  bin_to_zyz(bin, bw_out, z);
  zyz_to_quat(z, q);
  quat_to_xyz(q, e);
  if (zyz) memcpy(zyz, z, sizeof(z));
  if (quat) memcpy(quat, q, sizeof(q));
  if (xyz) memcpy(xyz, e, sizeof(e));
  if (T12) xyz_to_transform(e, T12);
  return PHGPU_OK;
}

static void xyz_to_transform(const double* e, float* T12) {
  {
    // RotateAroundXYZ: Rx(a) * Ry(b) * Rz(c) in float (rotation-utils.cc:17-24,109-143);
    // float cos / sin correctly rounded (double evaluation, one rounding), as
    // the device pose kernel (k_pose.cu) computes them
    const float a = (float)e[0], bb = (float)e[1], c = (float)e[2];
    const float ca = (float)cos((double)a), sa = (float)sin((double)a), cb = (float)cos((double)bb),
                sb = (float)sin((double)bb), cc = (float)cos((double)c), sc = (float)sin((double)c);
    const float X[3][3] = {{1, 0, 0}, {0, ca, -sa}, {0, sa, ca}};
    const float Y[3][3] = {{cb, 0, sb}, {0, 1, 0}, {-sb, 0, cb}};
    const float Z[3][3] = {{cc, sc, 0}, {-sc, cc, 0}, {0, 0, 1}};
    float XY[3][3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        float s = 0.0f;
        for (int k = 0; k < 3; ++k) s += X[i][k] * Y[k][j];
        XY[i][j] = s;
      }
    for (int i = 0; i < 3; ++i) {
      for (int j = 0; j < 3; ++j) {
        float s = 0.0f;
        for (int k = 0; k < 3; ++k) s += XY[i][k] * Z[k][j];
        T12[4 * i + j] = s;
      }
      T12[4 * i + 3] = 0.0f;
    }
  }
}

// Cyclic Jacobi eigen-decomposition of a symmetric 4x4 matrix (FP64):
// eigenvalues in w[i], eigenvectors in the columns of V (V[r * 4 + i]).
static void jacobi_eig4(const double* A0, double* w, double* V) {
  double A[16];
  memcpy(A, A0, sizeof(A));
  for (int i = 0; i < 16; ++i) V[i] = (i % 5 == 0) ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 64; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < 4; ++p)
      for (int q = p + 1; q < 4; ++q) off += A[p * 4 + q] * A[p * 4 + q];
    if (off < 1e-300) break;
    for (int p = 0; p < 4; ++p)
      for (int q = p + 1; q < 4; ++q) {
        const double apq = A[p * 4 + q];
        if (fabs(apq) < 1e-300) continue;
        const double theta = (A[q * 4 + q] - A[p * 4 + p]) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0), sn = t * c;
        for (int k = 0; k < 4; ++k) {  // A = A J (columns p, q)
          const double akp = A[k * 4 + p], akq = A[k * 4 + q];
          A[k * 4 + p] = c * akp - sn * akq;
          A[k * 4 + q] = sn * akp + c * akq;
        }
        for (int k = 0; k < 4; ++k) {  // A = J^T A (rows p, q)
          const double apk = A[p * 4 + k], aqk = A[q * 4 + k];
          A[p * 4 + k] = c * apk - sn * aqk;
          A[q * 4 + k] = sn * apk + c * aqk;
        }
        for (int k = 0; k < 4; ++k) {
          const double vkp = V[k * 4 + p], vkq = V[k * 4 + q];
          V[k * 4 + p] = c * vkp - sn * vkq;
          V[k * 4 + q] = sn * vkp + c * vkq;
        }
      }
  }
  for (int i = 0; i < 4; ++i) w[i] = A[i * 5];
}

void phgpu_peak_window(uint32_t index, uint32_t n, uint32_t k, uint32_t* first, uint32_t* count) {
  const uint32_t start = k > index ? index : index - k;
  const uint64_t hi = (uint64_t)index + k;
  const uint32_t end = hi >= n ? index : (uint32_t)hi;
  if (first) *first = start;
  if (count) *count = end - start + 1u;
}

int phgpu_bingham_peak(const double* values, uint32_t first_bin, uint32_t count, uint32_t bw_out, double* mode4,
                       double* omega4, double* xyz3) {
  if (!values || count == 0 || bw_out == 0) return PHGPU_ERR_INVALID;
  double wsum = 0.0;
  for (uint32_t i = 0; i < count; ++i) wsum += values[i];
  if (count > 1 && !(wsum > 0.0)) return PHGPU_ERR_INVALID;
  double C[16] = {0.0};
  for (uint32_t i = 0; i < count; ++i) {
    double z[3], q[4];
    bin_to_zyz(first_bin + i, bw_out, z);
    zyz_to_quat(z, q);
    const double w = count > 1 ? values[i] / wsum : values[i];
    for (int r = 0; r < 4; ++r)
      for (int c = 0; c < 4; ++c) C[r * 4 + c] += w * q[r] * q[c];
  }
  double ev[4], V[16];
  jacobi_eig4(C, ev, V);
  int order[4] = {0, 1, 2, 3};
  std::sort(order, order + 4, [&](int a, int b) { return ev[a] < ev[b]; });
  const int top = order[3];
  double m[4] = {V[0 * 4 + top], V[1 * 4 + top], V[2 * 4 + top], V[3 * 4 + top]};
  const double nrm = sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2] + m[3] * m[3]);
  const double sg = m[0] < 0 ? -1.0 : 1.0;
  for (int r = 0; r < 4; ++r) m[r] *= sg / nrm;
  double esum = 0.0;
  for (int i = 0; i < 4; ++i) esum += ev[i];
  if (mode4) memcpy(mode4, m, sizeof(m));
  if (omega4)
    for (int i = 0; i < 4; ++i) omega4[i] = esum != 0.0 ? ev[order[i]] / esum : 0.0;
  if (xyz3) quat_to_xyz(m, xyz3);
  return PHGPU_OK;
}

int phgpu_gaussian_peak(const double* values, uint32_t first_voxel, uint32_t count, uint32_t n_voxels,
                        int32_t lower, int32_t upper, double* mean3, double* cov9) {
  if (!values || count == 0 || n_voxels == 0) return PHGPU_ERR_INVALID;
  double wsum = 0.0;
  for (uint32_t i = 0; i < count; ++i) wsum += values[i];
  if (!(wsum > 0.0)) return PHGPU_ERR_INVALID;
  std::vector<double> t(3 * (size_t)count);
  double mu[3] = {0.0, 0.0, 0.0};
  for (uint32_t i = 0; i < count; ++i) {
    const uint32_t v = first_voxel + i, N = n_voxels;
    // Ind2Sub(i, N, N) (signal-utils.cc:5-19)
    const uint32_t sub[3] = {(v / N) % N, v % N, v / (N * N)};
    const double w = values[i] / wsum;
    for (int a = 0; a < 3; ++a) {
      t[3 * i + a] = phgpu_translation_from_index((double)sub[a], N, lower, upper);
      mu[a] += w * t[3 * i + a];
    }
  }
  // the reference scales the centred samples by sqrt(w) (a negative weight
  // gives NaN there, and here)
  double cov[9] = {0.0};
  for (uint32_t i = 0; i < count; ++i) {
    const double sw = sqrt(values[i] / wsum);
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) cov[r * 3 + c] += (sw * (t[3 * i + r] - mu[r])) * (sw * (t[3 * i + c] - mu[c]));
  }
  if (mean3) memcpy(mean3, mu, sizeof(mu));
  if (cov9) memcpy(cov9, cov, sizeof(cov));
  return PHGPU_OK;
}

double phgpu_translation_from_index(double index, uint32_t n_voxels, int32_t lower, int32_t upper) {
  if (index == 0) return 0.0;
  const double half = n_voxels / 2.0;
  const double width = (double)(abs(lower) + abs(upper) + 1);
  if (index <= half) return index * width / n_voxels;
  return (index - n_voxels) * width / n_voxels;
}

// ------------------------------------------------------------------ profiler

static cudaEvent_t pool_event(phgpu_ctx* c) {
  if (!c->ev_pool.empty()) {
    cudaEvent_t e = c->ev_pool.back();
    c->ev_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

ProfScope::ProfScope(phgpu_ctx* ctx, cudaStream_t st, int stg) : c(ctx), s(st), stage(stg) {
  if (c->prof_on) {
    a = pool_event(c);
    cudaEventRecord(a, s);
  }
}

ProfScope::~ProfScope() {
  if (!a) return;
  cudaEvent_t b = pool_event(c);
  cudaEventRecord(b, s);
  c->prof_recs.push_back(ProfRec{stage, a, b});
}

static const char* kStageNames[PS_COUNT] = {"upload", "s2_sample", "sht", "fuse_s2", "so3_synth",
                                            "so3_fft", "voxelize", "spatial_fwd", "fuse_z", "spatial_inv"};

int phgpu_profile_enable(phgpu_ctx* ctx, int enable) {
  if (!ctx) return PHGPU_ERR_INVALID;
  ctx->prof_on = enable != 0;
  ctx->prof_serial = enable == 2;
  return PHGPU_OK;
}

int phgpu_profile_read(phgpu_ctx* ctx, double* ms, unsigned long long* calls, int n) {
  if (!ctx) return PHGPU_ERR_INVALID;
  cudaSetDevice(ctx->prm.device);
  CK(cudaStreamSynchronize(ctx->s0));
  CK(cudaStreamSynchronize(ctx->s1));
  for (const ProfRec& r : ctx->prof_recs) {
    float t = 0.0f;
    if (cudaEventElapsedTime(&t, r.a, r.b) == cudaSuccess) {
      ctx->prof_ms[r.stage] += t;
      ctx->prof_n[r.stage] += 1;
    }
    ctx->ev_pool.push_back(r.a);
    ctx->ev_pool.push_back(r.b);
  }
  ctx->prof_recs.clear();
  for (int i = 0; i < n && i < PS_COUNT; ++i) {
    if (ms) ms[i] = ctx->prof_ms[i];
    if (calls) calls[i] = ctx->prof_n[i];
    ctx->prof_ms[i] = 0.0;
    ctx->prof_n[i] = 0;
  }
  return PHGPU_OK;
}

const char* phgpu_profile_stage_name(int stage) {
  return (stage >= 0 && stage < PS_COUNT) ? kStageNames[stage] : "";
}

int phgpu_profile_stage_count(void) { return PS_COUNT; }

unsigned long long phgpu_launch_count(void) { return g_launch_count.load(); }

unsigned long long phgpu_pose_reruns(const phgpu_ctx* ctx) { return ctx ? ctx->pose_reruns : 0ull; }

// ------------------------------------------------------------------ context

int phgpu_params_default(phgpu_params* p) {
  if (!p) return PHGPU_ERR_INVALID;
  memset(p, 0, sizeof(*p));
  p->spherical_bandwidth = 75;
  p->spherical_zero_padding = 0;
  p->spatial_n_voxels = 100;
  p->spatial_discretize_lower = -50;
  p->spatial_discretize_upper = 50;
  p->spatial_zero_padding = 0;
  p->spatial_low_pass_lower = 0.0f;
  p->spatial_low_pass_upper = 100000.0f;
  p->n_channels = 4;
  p->fusion_levels = 5;
  p->spherical_fusion = PHGPU_FUSION_LAPLACE;
  p->spatial_fusion = PHGPU_FUSION_LAPLACE;
  p->max_points = 1u << 18;
  p->flags = 0;
  p->device = 0;
  p->rot_peak_neighbors = 0;
  p->trans_peak_neighbors = 0;
  p->spherical_low_pass_lower = 0;
  p->spherical_low_pass_upper = 100000;
  p->precision = PHGPU_PRECISION_FP32;
  return PHGPU_OK;
}

const char* phgpu_last_error(const phgpu_ctx* ctx) {
  return ctx ? ctx->err.c_str() : g_create_error.c_str();
}

void* phgpu_stream(phgpu_ctx* ctx) { return ctx ? (void*)ctx->s0 : nullptr; }

uint32_t phgpu_sph_bandwidth(const phgpu_ctx* ctx) { return ctx ? (uint32_t)ctx->bw_out : 0u; }
uint32_t phgpu_spatial_correlation_size(const phgpu_ctx* ctx) { return ctx ? ctx->corr_size : 0u; }

template <typename T>
static int dalloc(phgpu_ctx* ctx, T** p, size_t bytes) {
  if (bytes == 0) bytes = 256;
  cudaError_t e = cudaMalloc((void**)p, bytes);
  if (e != cudaSuccess) {
    ctx->err = "cudaMalloc(" + std::to_string(bytes) + ") failed: " + cudaGetErrorString(e);
    *p = nullptr;
    return PHGPU_ERR_MEMORY;
  }
  ctx->allocs.push_back((void*)*p);
  ctx->device_bytes += bytes;
  return PHGPU_OK;
}

static void dfree(phgpu_ctx* ctx, void* p) {
  if (!p) return;
  auto it = std::find(ctx->allocs.begin(), ctx->allocs.end(), p);
  if (it != ctx->allocs.end()) ctx->allocs.erase(it);
  cudaFree(p);
}

static int ensure_cloud_capacity(phgpu_ctx* ctx, uint32_t n) {
  if (n <= ctx->cap_points) return PHGPU_OK;
  uint32_t cap = std::max<uint32_t>(n, ctx->cap_points * 2);
  for (int s = 0; s < 2; ++s) {
    dfree(ctx, ctx->d_xyzi[s]);
    dfree(ctx, ctx->d_refl[s]);
    dfree(ctx, ctx->d_amb[s]);
    dfree(ctx, ctx->d_sample_scratch[s]);
    dfree(ctx, ctx->d_lin[s]);
    CKV(dalloc(ctx, &ctx->d_xyzi[s], sizeof(float4) * cap));
    CKV(dalloc(ctx, &ctx->d_refl[s], sizeof(float) * cap));
    CKV(dalloc(ctx, &ctx->d_amb[s], sizeof(float) * cap));
    CKV(dalloc(ctx, &ctx->d_sample_scratch[s], sampler_scratch_bytes((int)cap, 4 * ctx->bw * ctx->bw)));
    CKV(dalloc(ctx, &ctx->d_lin[s], sizeof(uint32_t) * cap));
  }
  ctx->cap_points = cap;
  return PHGPU_OK;
}

int phgpu_ctx_create(const phgpu_params* prm, phgpu_ctx** out) { return phgpu_ctx_create_internal(prm, out, true); }

int phgpu_ctx_create_internal(const phgpu_params* prm, phgpu_ctx** out, bool wigner_table) {
  if (!prm || !out) {
    g_create_error = "null argument";
    return PHGPU_ERR_INVALID;
  }
  *out = nullptr;
  const int bw = (int)prm->spherical_bandwidth;
  const int bw_out = bw + (int)prm->spherical_zero_padding;
  const int N = (int)prm->spatial_n_voxels;
  if (bw < 2 || bw > 512 || N < 1 || N > 1024 || (uint64_t)N + 2ull * prm->spatial_zero_padding > 1024 ||
      prm->n_channels < 1 || prm->n_channels > 4 || prm->fusion_levels < 1 ||
      prm->fusion_levels > (uint32_t)kMaxLevels || prm->spherical_fusion > PHGPU_FUSION_MIX || prm->spatial_fusion > PHGPU_FUSION_LOW_PASS ||
      prm->precision > PHGPU_PRECISION_BF16X3) {
    g_create_error =
        "unsupported configuration (2 <= bandwidth <= 512, 1 <= n_voxels + 2 spatial zero padding <= 1024, "
        "1..4 channels, 1..8 fusion levels, spherical fusion 0..3, spatial fusion 0..2, precision 0..2)";
    return PHGPU_ERR_INVALID;
  }
  phgpu_ctx* ctx = new phgpu_ctx();
  ctx->prm = *prm;
  ctx->own_wigner_table = wigner_table;
  ctx->bw = bw;
  ctx->bw_out = bw_out;
  ctx->N = N;
  ctx->pad = (int)prm->spatial_zero_padding;
  ctx->M = N + 2 * ctx->pad;
  {
    // SpatialCorrelation's constructor (spatial-correlation.cc:17-25): the
    // padded size in double, truncated (M^3 - 1 for many N, pad)
    const double ratio = (double)(uint32_t)ctx->M / (double)N;
    const double factor = ratio * ratio * ratio;
    const uint32_t nv = (uint32_t)N * (uint32_t)N * (uint32_t)N;
    ctx->corr_size = ctx->pad ? (uint32_t)((double)nv * factor) : nv;
  }
  if (cudaSetDevice(prm->device) != cudaSuccess) {
    g_create_error = "cudaSetDevice failed";
    delete ctx;
    return PHGPU_ERR_CUDA;
  }
  int rc = phgpu_ctx_init(ctx);
  if (rc != PHGPU_OK) {
    g_create_error = ctx->err;
    phgpu_ctx_destroy(ctx);
    return rc;
  }
  *out = ctx;
  return PHGPU_OK;
}

int phgpu_ctx_init(phgpu_ctx* ctx) {
  const phgpu_params* prm = &ctx->prm;
  const int bw = ctx->bw, bw_out = ctx->bw_out, N = ctx->N;
  CK(cudaStreamCreateWithFlags(&ctx->s0, cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&ctx->s1, cudaStreamNonBlocking));
  CK(cudaEventCreateWithFlags(&ctx->ev_a, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&ctx->ev_b, cudaEventDisableTiming));
  CK(spatial_init_attributes());
  CK(so3_init_attributes());
  CK(sht_init_attributes());
  std::string perr;
  if (!make_fft_plan(2 * bw, &ctx->plan_s2, &ctx->d_tw[0], &perr) ||
      !make_fft_plan(2 * bw_out, &ctx->plan_so3, &ctx->d_tw[1], &perr) ||
      !make_fft_plan(N, &ctx->plan_sp, &ctx->d_tw[2], &perr)) {
    ctx->err = perr;
    return PHGPU_ERR_INVALID;
  }
  if (spatial_slab_path(N)) {
    if (!make_fft_plan(N / 2, &ctx->plan_sp_half, &ctx->d_tw[3], &perr)) {
      ctx->err = perr;
      return PHGPU_ERR_INVALID;
    }
    ctx->has_sp_half = true;
  }
  if (ctx->pad) {
    if (!make_fft_plan(ctx->M, &ctx->plan_pad, &ctx->d_tw_pad[0], &perr)) {
      ctx->err = perr;
      return PHGPU_ERR_INVALID;
    }
    if (spatial_slab_path(ctx->M)) {
      if (!make_fft_plan(ctx->M / 2, &ctx->plan_pad_half, &ctx->d_tw_pad[1], &perr)) {
        ctx->err = perr;
        return PHGPU_ERR_INVALID;
      }
      ctx->has_pad_half = true;
    }
  }
  ctx->bands_s2 = make_bands((uint32_t)(bw * bw), (int)prm->fusion_levels, 4.0f);
  ctx->bands_sp = make_bands((uint32_t)N * (uint32_t)N * (uint32_t)N, (int)prm->fusion_levels, 4.0f);
  // DH grid directions (spherical-sampler.cc:29-64), float sin/cos of float angles
  const int n = 2 * bw;
  std::vector<float4> grid((size_t)n * n);
  for (int i = 0; i < n; ++i) {
    const float th = (float)((M_PI * (double)(2 * i + 1)) / (double)(4 * bw));
    for (int j = 0; j < n; ++j) {
      const float ph = (float)((2.0 * M_PI * (double)j) / (double)(2 * bw));
      const float dist = 1.0f;
      grid[(size_t)i * n + j] = make_float4(dist * sinf(th) * cosf(ph), dist * sinf(th) * sinf(ph),
                                            dist * cosf(th), 0.0f);
    }
  }
  CKV(dalloc(ctx, &ctx->d_grid, sizeof(float4) * grid.size()));
  CK(cudaMemcpy(ctx->d_grid, grid.data(), sizeof(float4) * grid.size(), cudaMemcpyHostToDevice));
  // Driscoll-Healy weights (lib/SOFT/makeweights.c:68-91 behaviour)
  std::vector<double> w(n);
  for (int k = 0; k < n; ++k) {
    const double th = M_PI * (2.0 * k + 1.0) / (4.0 * bw);
    double s = 0.0;
    for (int i = 0; i < bw; ++i) s += sin((2.0 * i + 1.0) * th) / (2.0 * i + 1.0);
    w[k] = (2.0 / (double)bw) * sin(th) * s;
  }
  CKV(dalloc(ctx, &ctx->d_weights, sizeof(double) * n));
  CK(cudaMemcpy(ctx->d_weights, w.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
  CKV(dalloc(ctx, &ctx->d_legendre, sizeof(float) * legendre_table_entries(bw)));
  CK(launch_legendre_table(bw, ctx->d_weights, ctx->d_legendre, ctx->s0));
  if (prm->precision != PHGPU_PRECISION_FP32) {
    if (!sht_leg_tc_supported(bw, 1, (int)prm->precision)) {
      ctx->err = "the tensor-core Legendre contraction supports bandwidths <= 256";
      return PHGPU_ERR_INVALID;
    }
    CKV(dalloc(ctx, &ctx->d_legendre_tc, sizeof(float) * legendre_tc_floats(bw)));
    CK(launch_legendre_tc_layout(bw, ctx->d_legendre, ctx->d_legendre_tc, ctx->s0));
  }
  // histc edges (phase-aligner.cc:27-30): float LinSpaced of Eigen >= 3.3,
  // which counts down from the high end when |hi| < |lo|
  std::vector<float> e(N);
  const float flo = (float)prm->spatial_discretize_lower, fhi = (float)prm->spatial_discretize_upper;
  const float step = (N == 1) ? 0.0f : (fhi - flo) / (float)(N - 1);
  const bool flip = fabsf(fhi) < fabsf(flo);
  for (int i = 0; i < N; ++i) {
    if (flip)
      e[i] = (i == 0) ? flo : (fhi - (float)(N - 1 - i) * step);
    else
      e[i] = (i == N - 1) ? fhi : (flo + (float)i * step);
  }
  CKV(dalloc(ctx, &ctx->d_edges, sizeof(float) * N));
  CK(cudaMemcpy(ctx->d_edges, e.data(), sizeof(float) * N, cudaMemcpyHostToDevice));
  // squared voxel size of the sampler rejection (point-cloud.cc:66-72)
  const float vs = (fabsf(prm->spatial_low_pass_lower) + fabsf(prm->spatial_low_pass_upper)) /
                   (float)prm->spatial_n_voxels;
  ctx->max_sq = vs * vs;
  // buffers
  const size_t nq = (size_t)4 * bw * bw;
  CKV(dalloc(ctx, &ctx->d_samples, sizeof(float) * 2 * 4 * nq));
  CK(cudaMemset(ctx->d_samples, 0, sizeof(float) * 2 * 4 * nq));
  if (prm->spherical_fusion == PHGPU_FUSION_MIX) CKV(dalloc(ctx, &ctx->d_mix, sizeof(float) * 2 * nq));
  for (int s = 0; s < 2; ++s) CKV(dalloc(ctx, &ctx->d_nn[s], sizeof(int32_t) * nq));
  CKV(dalloc(ctx, &ctx->d_coef, sizeof(float2) * 8 * bw * bw));
  CKV(dalloc(ctx, &ctx->d_fphi, sizeof(float2) * sht_scratch_entries(bw)));
  CKV(dalloc(ctx, &ctx->d_fused, sizeof(float2) * 2 * bw * (2 * bw - 1)));
  CK(cudaMemset(ctx->d_fused, 0, sizeof(float2) * 2 * bw * (2 * bw - 1)));
  const size_t no = (size_t)2 * bw_out;
  CKV(dalloc(ctx, &ctx->d_S, sizeof(float2) * no * no * bw_out));
  CK(cudaMemset(ctx->d_S, 0, sizeof(float2) * no * no * bw_out));
  {
    std::vector<double> bt(3 * (size_t)no);
    so3_beta_table(bw_out, bt.data());
    CKV(dalloc(ctx, &ctx->d_beta_tab, sizeof(double) * bt.size()));
    CK(cudaMemcpy(ctx->d_beta_tab, bt.data(), sizeof(double) * bt.size(), cudaMemcpyHostToDevice));
    std::vector<double> wt;
    so3_wigner_table(bw, wt);
    CKV(dalloc(ctx, &ctx->d_wig_tab, sizeof(double) * wt.size()));
    CK(cudaMemcpy(ctx->d_wig_tab, wt.data(), sizeof(double) * wt.size(), cudaMemcpyHostToDevice));
  }
  if (prm->precision != PHGPU_PRECISION_FP32 && ctx->own_wigner_table) {
    // tensor-core synthesis: the Wigner-d table, generated once in FP64
    if (!so3_tc_supported(bw_out, 1, (int)prm->precision)) {
      ctx->err = "the tensor-core SO(3) synthesis supports bandwidth + spherical zero padding <= 256";
      return PHGPU_ERR_INVALID;
    }
    std::vector<size_t> off;
    const size_t nf = so3_table_layout(bw, bw_out, &off);
    CKV(dalloc(ctx, &ctx->d_class_off, sizeof(size_t) * off.size()));
    CK(cudaMemcpy(ctx->d_class_off, off.data(), sizeof(size_t) * off.size(), cudaMemcpyHostToDevice));
    CKV(dalloc(ctx, &ctx->d_wtable, sizeof(float) * nf));
    CK(launch_so3_table(bw, bw_out, ctx->d_beta_tab, ctx->d_wig_tab, ctx->d_class_off, ctx->d_wtable, ctx->s0));
  }
  const size_t nv = (size_t)N * N * N;
  const size_t H = (size_t)N * N * spatial_h2p(N);
  for (int s = 0; s < 2; ++s) {
    CKV(dalloc(ctx, &ctx->d_grids[s], sizeof(float) * 5 * nv));
    CKV(dalloc(ctx, &ctx->d_rowlive[s], (size_t)N * N));
  }
  CKV(dalloc(ctx, &ctx->d_slab_nz, (size_t)8 * N));
  CK(cudaMemset(ctx->d_slab_nz, 1, (size_t)8 * N));  // nothing known to be zero yet
  CKV(dalloc(ctx, &ctx->d_spec, sizeof(float2) * 8 * H));
  CKV(dalloc(ctx, &ctx->d_cspec, sizeof(float2) * H));
  // volumes: kept on request, and needed by the peak-neighbourhood fits
  if ((prm->flags & PHGPU_FLAG_KEEP_VOLUMES) || prm->rot_peak_neighbors > 0)
    CKV(dalloc(ctx, &ctx->d_rotvol, sizeof(float) * no * no * no));
  if ((prm->flags & PHGPU_FLAG_KEEP_VOLUMES) || prm->trans_peak_neighbors > 0)
    CKV(dalloc(ctx, &ctx->d_transvol, sizeof(float) * (ctx->pad ? (size_t)ctx->M * ctx->M * ctx->M : nv)));
  if (ctx->pad) {
    const size_t HM = (size_t)ctx->M * ctx->M * spatial_h2p(ctx->M);
    CKV(dalloc(ctx, &ctx->d_cspec_pad, sizeof(float2) * HM));
    if (prm->spatial_fusion == PHGPU_FUSION_LAPLACE)
      for (int s = 0; s < 2; ++s) CKV(dalloc(ctx, &ctx->d_prev[s], sizeof(float2) * H));
  }
  // [0] rotation argmax, [1] translation argmax, [2] kernel status bits (sticky)
  CKV(dalloc(ctx, &ctx->d_argmax, sizeof(unsigned long long) * 3));
  CK(cudaMemset(ctx->d_argmax, 0, sizeof(unsigned long long) * 3));
  CK(cudaMallocHost((void**)&ctx->h_argmax, sizeof(unsigned long long) * 3));
  CKV(dalloc(ctx, &ctx->d_T, sizeof(float) * 16));
  CK(cudaMallocHost((void**)&ctx->h_T, sizeof(float) * 16));
  CKV(dalloc(ctx, &ctx->d_np, sizeof(uint32_t) * 2));
  CK(cudaMemset(ctx->d_np, 0, sizeof(uint32_t) * 2));
  CK(cudaMallocHost((void**)&ctx->h_np, sizeof(uint32_t) * 2));
  ctx->h_argmax[0] = ctx->h_argmax[1] = ctx->h_argmax[2] = 0ull;
  CKV(ensure_cloud_capacity(ctx, prm->max_points ? prm->max_points : (1u << 18)));
  CK(cudaStreamSynchronize(ctx->s0));
  return PHGPU_OK;
}

int phgpu_ctx_destroy(phgpu_ctx* ctx) {
  if (!ctx) return PHGPU_OK;
  cudaSetDevice(ctx->prm.device);
  if (ctx->s0) cudaStreamSynchronize(ctx->s0);
  if (ctx->s1) cudaStreamSynchronize(ctx->s1);
  for (void* p : ctx->allocs) cudaFree(p);
  ctx->allocs.clear();
  for (int i = 0; i < 4; ++i)
    if (ctx->d_tw[i]) cudaFree(ctx->d_tw[i]);
  for (int i = 0; i < 2; ++i)
    if (ctx->d_tw_pad[i]) cudaFree(ctx->d_tw_pad[i]);
  if (ctx->h_argmax) cudaFreeHost(ctx->h_argmax);
  if (ctx->h_T) cudaFreeHost(ctx->h_T);
  if (ctx->h_np) cudaFreeHost(ctx->h_np);
  for (const ProfRec& r : ctx->prof_recs) {
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  for (cudaEvent_t e : ctx->ev_pool) cudaEventDestroy(e);
  if (ctx->ev_a) cudaEventDestroy(ctx->ev_a);
  if (ctx->ev_b) cudaEventDestroy(ctx->ev_b);
  if (ctx->s0) cudaStreamDestroy(ctx->s0);
  if (ctx->s1) cudaStreamDestroy(ctx->s1);
  delete ctx;
  return PHGPU_OK;
}

// ------------------------------------------------------------------ stages

int phgpu_upload_cloud(phgpu_ctx* ctx, const phgpu_cloud* c, int side, cudaStream_t st) {
  CKV(ensure_cloud_capacity(ctx, c->n_points));
  const cudaMemcpyKind kind = c->on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  if (c->n_points) {
    CK(cudaMemcpyAsync(ctx->d_xyzi[side], c->xyzi, sizeof(float4) * c->n_points, kind, st));
    if (c->reflectivity)
      CK(cudaMemcpyAsync(ctx->d_refl[side], c->reflectivity, sizeof(float) * c->n_points, kind, st));
    if (c->ambient)
      CK(cudaMemcpyAsync(ctx->d_amb[side], c->ambient, sizeof(float) * c->n_points, kind, st));
  }
  ctx->np[side] = c->n_points;
  ctx->has_refl[side] = c->reflectivity != nullptr;
  ctx->has_amb[side] = c->ambient != nullptr;
  if (ctx->dev_counts) {
    ctx->h_np[side] = c->n_points;
    CK(cudaMemcpyAsync(ctx->d_np + side, ctx->h_np + side, sizeof(uint32_t), cudaMemcpyHostToDevice, st));
  }
  return PHGPU_OK;
}

static int run_sample(phgpu_ctx* ctx, int side, cudaStream_t st) {
  SampleArgs a;
  a.xyzi = ctx->d_xyzi[side];
  a.refl = ctx->has_refl[side] ? ctx->d_refl[side] : nullptr;
  a.amb = ctx->has_amb[side] ? ctx->d_amb[side] : nullptr;
  a.n_points = ctx->dev_counts ? (int)ctx->cap_points : (int)ctx->np[side];
  a.n_dev = ctx->dev_counts ? ctx->d_np + side : nullptr;
  a.max_points = (int)ctx->cap_points;
  a.grid = ctx->d_grid;
  a.n_queries = 4 * ctx->bw * ctx->bw;
  a.n2b = 2 * ctx->bw;
  a.max_sq = ctx->max_sq;
  a.n_out_ch = 4;
  a.out = ctx->d_samples + (size_t)side * 4 * a.n_queries;
  a.nn_idx = ctx->d_nn[side];
  a.scratch = ctx->d_sample_scratch[side];
  {
    ProfScope ps(ctx, st, PS_SAMPLE);
    CK(launch_sample(a, st));
  }
  ctx->sampled[side] = true;
  return PHGPU_OK;
}

int phgpu_sample_s2(phgpu_ctx* ctx, const phgpu_cloud* cloud, int side) {
  if (!ctx || !cloud || side < 0 || side > 1) return PHGPU_ERR_INVALID;
  cudaSetDevice(ctx->prm.device);
  CKV(phgpu_upload_cloud(ctx, cloud, side, ctx->s0));
  CKV(run_sample(ctx, side, ctx->s0));
  CK(cudaStreamSynchronize(ctx->s0));
  return PHGPU_OK;
}

int phgpu_get_samples(phgpu_ctx* ctx, int side, double* values, int32_t* nn_index) {
  if (!ctx || side < 0 || side > 1) return PHGPU_ERR_INVALID;
  if (!ctx->sampled[side]) {
    ctx->err = "no samples for this side";
    return PHGPU_ERR_STATE;
  }
  cudaSetDevice(ctx->prm.device);
  const size_t nq = (size_t)4 * ctx->bw * ctx->bw;
  if (values) {
    std::vector<float> tmp(4 * nq);
    CK(cudaMemcpy(tmp.data(), ctx->d_samples + (size_t)side * 4 * nq, sizeof(float) * 4 * nq,
                  cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < 4 * nq; ++i) values[i] = tmp[i];
  }
  if (nn_index) CK(cudaMemcpy(nn_index, ctx->d_nn[side], sizeof(int32_t) * nq, cudaMemcpyDeviceToHost));
  return PHGPU_OK;
}

// SO(3) launch arguments of this context alone (a batch of one request).
So3Args so3_args(phgpu_ctx* ctx) {
  So3Args o;
  memset(&o, 0, sizeof(o));
  o.bw_in = ctx->bw;
  o.bw_out = ctx->bw_out;
  o.beta_tab = ctx->d_beta_tab;
  o.wig_tab = ctx->d_wig_tab;
  o.plan = &ctx->plan_so3;
  o.batch.count = 1;
  o.batch.fused[0] = ctx->d_fused;
  o.batch.out[0].S = ctx->d_S;
  o.batch.out[0].argmax = ctx->d_argmax;
  o.batch.out[0].volume = ctx->d_rotvol;
  o.beta_tile = (int)ctx->tune.so3_beta_tile;
  o.tc_chunk = (int)ctx->tune.tc_chunk;
  return o;
}

So3Table so3_table(phgpu_ctx* ctx) {
  So3Table t;
  t.table = ctx->d_wtable;
  t.class_off = ctx->d_class_off;
  t.precision = (int)ctx->prm.precision;
  return t;
}

// Spherical correlation of the sample grids currently in d_samples.
// SHT of both sides' sample grids and their fusion (up to the fused spectra);
// resets the rotation argmax.
static ShtArgs sht_args(phgpu_ctx* ctx, int n_data, bool mix) {
  const size_t nq = (size_t)4 * ctx->bw * ctx->bw;
  ShtArgs s;
  s.bw = ctx->bw;
  s.n_data = mix ? 1 : n_data;
  s.side_stride = mix ? nq : 4 * nq;
  s.signal = mix ? ctx->d_mix : ctx->d_samples;
  s.plan = &ctx->plan_s2;
  s.table = ctx->d_legendre;
  s.fphi = ctx->d_fphi;
  s.coef = ctx->d_coef;
  if (ctx->prm.precision != PHGPU_PRECISION_FP32) {
    s.table_tc = ctx->d_legendre_tc;
    s.precision = (int)ctx->prm.precision;
    s.tc_chunk = (int)ctx->tune.tc_chunk;
    s.status = ctx->d_argmax + 2;
  }
  return s;
}

static FuseS2Args fuse_args(phgpu_ctx* ctx, int n_data, int n_total, int laplace) {
  const int bw = ctx->bw;
  FuseS2Args f;
  f.bw = bw;
  f.lowpass = (!laplace && ctx->prm.spherical_fusion == PHGPU_FUSION_LOW_PASS) ? 1 : 0;
  f.lp_lo = std::min<uint32_t>(ctx->prm.spherical_low_pass_lower, (uint32_t)(bw * bw));
  f.lp_hi = std::min<uint32_t>(ctx->prm.spherical_low_pass_upper, (uint32_t)(bw * bw));
  f.n_data_ch = n_data;
  f.n_total_ch = n_total;
  f.laplace = laplace;
  f.bands = ctx->bands_s2;
  f.coef = ctx->d_coef;
  f.fused = ctx->d_fused;
  return f;
}

// Sampled grids to the phi transform alone (the Legendre contraction and the
// fusion then run batched across a wave, phgpu_run_sph_leg_fuse_batch).
int phgpu_run_sph_phi(phgpu_ctx* ctx, int n_data, cudaStream_t st, bool mix) {
  const size_t nq = (size_t)4 * ctx->bw * ctx->bw;
  if (mix) CK(launch_mix_signal(ctx->d_samples, 4 * nq, (int)nq, ctx->d_mix, st));
  ProfScope ps(ctx, st, PS_SHT);
  CK(launch_sht_phi(sht_args(ctx, n_data, mix), st));
  return PHGPU_OK;
}

int phgpu_run_sph_leg_fuse_batch(phgpu_ctx* const* ctx, int k, int n_data, int n_total, int laplace, bool mix,
                                 cudaStream_t st) {
  phgpu_ctx* c0 = ctx[0];
  if (k < 1 || k > kMaxWave || c0->prm.precision == PHGPU_PRECISION_FP32) return PHGPU_ERR_INVALID;
  const ShtArgs s = sht_args(c0, n_data, mix);
  ShtBatch b;
  b.count = k;
  for (int i = 0; i < k; ++i) {
    b.fphi[i] = ctx[i]->d_fphi;
    b.coef[i] = ctx[i]->d_coef;
  }
  {
    ProfScope ps(c0, st, PS_SHT);
    CKC(c0, launch_sht_leg_tc(s.bw, s.n_data, b, s.table_tc, s.precision, s.tc_chunk, s.status, st));
  }
  FuseS2Args f = fuse_args(c0, mix ? 1 : n_data, n_total, laplace);
  f.count = k;
  for (int i = 0; i < k; ++i) {
    f.coef_b[i] = ctx[i]->d_coef;
    f.fused_b[i] = ctx[i]->d_fused;
  }
  {
    ProfScope ps(c0, st, PS_FUSE_S2);
    CKC(c0, launch_fuse_s2(f, st));
  }
  for (int i = 0; i < k; ++i) CKC(c0, cudaMemsetAsync(ctx[i]->d_argmax, 0, sizeof(unsigned long long), st));
  return PHGPU_OK;
}

int phgpu_run_sph_front(phgpu_ctx* ctx, int n_data, int n_total, int laplace, cudaStream_t st, bool mix) {
  const size_t nq = (size_t)4 * ctx->bw * ctx->bw;
  if (mix) CK(launch_mix_signal(ctx->d_samples, 4 * nq, (int)nq, ctx->d_mix, st));
  {
    ProfScope ps(ctx, st, PS_SHT);
    CK(launch_sht(sht_args(ctx, n_data, mix), st));
  }
  {
    ProfScope ps(ctx, st, PS_FUSE_S2);
    CK(launch_fuse_s2(fuse_args(ctx, n_data, n_total, laplace), st));
  }
  CK(cudaMemsetAsync(ctx->d_argmax, 0, sizeof(unsigned long long), st));
  return PHGPU_OK;
}

// SO(3) synthesis, angle transforms and argmax of the fused spectra of
// ctx[0..k) (one shape) on stream st: one batched launch per stage.  The
// tensor-core synthesis reads `table` (null: the FP32 synthesis).
int phgpu_run_so3_batch(phgpu_ctx* const* ctx, int k, const So3Table* table, cudaStream_t st) {
  if (k < 1 || k > kMaxWave) return PHGPU_ERR_INVALID;
  So3Args o = so3_args(ctx[0]);
  o.batch.count = k;
  for (int i = 0; i < k; ++i) {
    o.batch.fused[i] = ctx[i]->d_fused;
    o.batch.out[i].S = ctx[i]->d_S;
    o.batch.out[i].argmax = ctx[i]->d_argmax;
    o.batch.out[i].volume = ctx[i]->d_rotvol;
  }
  phgpu_ctx* c0 = ctx[0];
  {
    ProfScope ps(c0, st, PS_SO3_SYNTH);
    if (table) {
      if (launch_so3_synth_tc(o, *table, c0->d_argmax + 2, st) != cudaSuccess) {
        c0->err = "tensor-core SO(3) synthesis launch failed";
        return PHGPU_ERR_CUDA;
      }
    } else {
      CKC(c0, launch_so3_synth(o, st));
    }
  }
  {
    ProfScope ps(c0, st, PS_SO3_FFT);
    CKC(c0, launch_so3_fft(o, st));
  }
  for (int i = 0; i < k; ++i) ctx[i]->have_rot = true;
  return PHGPU_OK;
}

// Spherical correlation of the sample grids currently in d_samples; the bin
// and status are read back to h_argmax[0], [2].
int phgpu_run_sph(phgpu_ctx* ctx, int n_data, int n_total, int laplace, cudaStream_t st, bool mix) {
  CKV(phgpu_run_sph_front(ctx, n_data, n_total, laplace, st, mix));
  So3Table t = so3_table(ctx);
  CKV(phgpu_run_so3_batch(&ctx, 1, t.table ? &t : nullptr, st));
  CK(cudaMemcpyAsync(ctx->h_argmax, ctx->d_argmax, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(ctx->h_argmax + 2, ctx->d_argmax + 2, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
  return PHGPU_OK;
}

int phgpu_sph_correlate(phgpu_ctx* ctx, const double* const* f, const double* const* g, uint32_t C) {
  if (!ctx || !f || !g || C < 1 || C > 4) {
    if (ctx) ctx->err = "phgpu_sph_correlate: 1..4 channels required";
    return PHGPU_ERR_INVALID;
  }
  cudaSetDevice(ctx->prm.device);
  const size_t nq = (size_t)4 * ctx->bw * ctx->bw;
  std::vector<float> tmp(2 * 4 * nq, 0.0f);
  for (uint32_t c = 0; c < C; ++c)
    for (size_t i = 0; i < nq; ++i) {
      tmp[c * nq + i] = (float)f[c][i];
      tmp[4 * nq + c * nq + i] = (float)g[c][i];
    }
  CK(cudaMemcpyAsync(ctx->d_samples, tmp.data(), sizeof(float) * tmp.size(), cudaMemcpyHostToDevice, ctx->s0));
  const int laplace = (C >= 2 && ctx->prm.spherical_fusion == PHGPU_FUSION_LAPLACE) ? 1 : 0;
  CKV(phgpu_run_sph(ctx, (int)C, (int)C, laplace, ctx->s0));
  CK(cudaStreamSynchronize(ctx->s0));
  return PHGPU_OK;
}

int phgpu_sph_correlate_sampled(phgpu_ctx* ctx) {
  if (!ctx) return PHGPU_ERR_INVALID;
  if (!ctx->sampled[0] || !ctx->sampled[1]) {
    ctx->err = "both sides must be sampled first";
    return PHGPU_ERR_STATE;
  }
  cudaSetDevice(ctx->prm.device);
  const int nd = std::max(ctx->has_amb[0] || ctx->has_amb[1] ? 4 : 0,
                          ctx->has_refl[0] || ctx->has_refl[1] ? 3 : 2);
  const int laplace = ctx->prm.spherical_fusion == PHGPU_FUSION_LAPLACE ? 1 : 0;
  CKV(phgpu_run_sph(ctx, laplace ? nd : 1, (int)ctx->prm.n_channels, laplace, ctx->s0,
                    ctx->prm.spherical_fusion == PHGPU_FUSION_MIX));
  CK(cudaStreamSynchronize(ctx->s0));
  return PHGPU_OK;
}

int phgpu_sph_result(phgpu_ctx* ctx, uint32_t* bin, float* peak, double* corr_out) {
  if (!ctx) return PHGPU_ERR_INVALID;
  if (!ctx->have_rot) {
    ctx->err = "no spherical correlation computed";
    return PHGPU_ERR_STATE;
  }
  cudaSetDevice(ctx->prm.device);
  CK(cudaStreamSynchronize(ctx->s0));
  if (ctx->h_argmax[2] & 2ull) {
    ctx->err = "a wait in the tensor-core SO(3) synthesis timed out";
    return PHGPU_ERR_CUDA;
  }
  const unsigned long long k = ctx->h_argmax[0];
  if (bin) *bin = unpack_index(k);
  if (peak) *peak = float_from_order_bits((uint32_t)(k >> 32));
  if (corr_out) {
    if (!ctx->d_rotvol) {
      ctx->err = "volumes not kept (PHGPU_FLAG_KEEP_VOLUMES)";
      return PHGPU_ERR_STATE;
    }
    const size_t n = (size_t)8 * ctx->bw_out * ctx->bw_out * ctx->bw_out;
    std::vector<float> tmp(n);
    CK(cudaMemcpy(tmp.data(), ctx->d_rotvol, sizeof(float) * n, cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < n; ++i) corr_out[i] = tmp[i];
  }
  return PHGPU_OK;
}

// Spatial channel count with data: {intensity, range} always, + reflectivity, + ambient.
static int sp_channels(int has_refl, int has_amb) { return has_amb ? 4 : (has_refl ? 3 : 2); }

int phgpu_run_voxelize(phgpu_ctx* ctx, int side, const float* T12, int n_data, cudaStream_t st,
                       const float* T_dev) {
  const size_t nv = (size_t)ctx->N * ctx->N * ctx->N;
  if (ctx->clean_planes[side] < n_data + 1) {
    CK(cudaMemsetAsync(ctx->d_grids[side], 0, sizeof(float) * (n_data + 1) * nv, st));
    CK(cudaMemsetAsync(ctx->d_rowlive[side], 0, (size_t)ctx->N * ctx->N, st));
  }
  ctx->clean_planes[side] = 0;
  VoxelArgs v;
  v.xyzi = ctx->d_xyzi[side];
  v.refl = ctx->has_refl[side] ? ctx->d_refl[side] : nullptr;
  v.amb = ctx->has_amb[side] ? ctx->d_amb[side] : nullptr;
  v.n_points = ctx->dev_counts ? (int)ctx->cap_points : (int)ctx->np[side];
  v.n_dev = ctx->dev_counts ? ctx->d_np + side : nullptr;
  v.N = ctx->N;
  v.edges = ctx->d_edges;
  v.has_T = T12 ? 1 : 0;
  for (int i = 0; i < 12; ++i) v.T[i] = T12 ? T12[i] : 0.0f;
  v.n_data_ch = n_data;
  v.grids = ctx->d_grids[side];
  v.lin_out = ctx->d_lin[side];
  v.rowlive = ctx->d_rowlive[side];
  v.T_dev = T_dev;
  {
    ProfScope ps(ctx, st, PS_VOXELIZE);
    CK(launch_voxelize(v, st));
  }
  ctx->vox_ch[side] = n_data;
  ctx->voxelized[side] = true;
  ctx->grids_live[side] = true;
  return PHGPU_OK;
}

// After the forward transform of a voxelised side inside register_pair (the
// grids are internal there): zero what the voxelisation wrote, so the next
// voxelisation of this side needs no full-grid memset.
static int clear_voxelized(phgpu_ctx* ctx, int side, cudaStream_t st) {
  const int planes = ctx->vox_ch[side] + 1;
  const size_t nv = (size_t)ctx->N * ctx->N * ctx->N;
  CK(launch_clear_voxels(ctx->d_lin[side], ctx->dev_counts ? (int)ctx->cap_points : (int)ctx->np[side],
                         ctx->d_grids[side], nv, planes, ctx->d_rowlive[side], ctx->N, st,
                         ctx->dev_counts ? ctx->d_np + side : nullptr));
  ctx->clean_planes[side] = planes;
  ctx->grids_live[side] = false;
  return PHGPU_OK;
}

int phgpu_voxelize(phgpu_ctx* ctx, const phgpu_cloud* cloud, int side, const float* T12) {
  if (!ctx || !cloud || side < 0 || side > 1) return PHGPU_ERR_INVALID;
  cudaSetDevice(ctx->prm.device);
  CKV(phgpu_upload_cloud(ctx, cloud, side, ctx->s0));
  CKV(phgpu_run_voxelize(ctx, side, T12, 4, ctx->s0));
  CK(cudaStreamSynchronize(ctx->s0));
  return PHGPU_OK;
}

int phgpu_get_voxel_index(phgpu_ctx* ctx, int side, uint32_t* lin, uint32_t n_points) {
  if (!ctx || side < 0 || side > 1 || !lin) return PHGPU_ERR_INVALID;
  if (!ctx->voxelized[side] || n_points > ctx->np[side]) {
    ctx->err = "no voxelisation for this side / too many points requested";
    return PHGPU_ERR_STATE;
  }
  cudaSetDevice(ctx->prm.device);
  CK(cudaMemcpy(lin, ctx->d_lin[side], sizeof(uint32_t) * n_points, cudaMemcpyDeviceToHost));
  return PHGPU_OK;
}

static SpatialArgs spatial_args(phgpu_ctx* ctx, int n_data, int n_total, int laplace, int means) {
  SpatialArgs a;
  a.N = ctx->N;
  a.n_data_ch = n_data;
  a.n_total_ch = n_total;
  a.laplace = laplace;
  a.lowpass = (!laplace && ctx->prm.spatial_fusion == PHGPU_FUSION_LOW_PASS) ? 1 : 0;
  // the low-pass cube: [lower, min(upper, N)] (spatial-correlation-low-pass.cc:11-19)
  a.lp_lo = ctx->prm.spatial_low_pass_lower > 0.f ? (uint32_t)ctx->prm.spatial_low_pass_lower : 0u;
  a.lp_hi = std::min<uint32_t>(ctx->prm.spatial_low_pass_upper > 0.f ? (uint32_t)ctx->prm.spatial_low_pass_upper : 0u,
                               (uint32_t)ctx->N);
  a.bands = ctx->bands_sp;
  a.grids_f = ctx->d_grids[0];
  a.grids_g = ctx->d_grids[1];
  a.grids_are_means = means;
  // row flags describe voxelised grids only (host-written grids are dense)
  a.rowlive_f = means ? nullptr : ctx->d_rowlive[0];
  a.rowlive_g = means ? nullptr : ctx->d_rowlive[1];
  // the padded path transforms the spectra in place: no slab stays known-zero
  a.slab_nz = ctx->pad ? nullptr : ctx->d_slab_nz;
  a.spec = ctx->d_spec;
  a.cspec = ctx->d_cspec;
  a.plan = &ctx->plan_sp;
  a.plan_half = ctx->has_sp_half ? &ctx->plan_sp_half : nullptr;
  a.argmax = ctx->d_argmax + 1;
  a.status = ctx->d_argmax + 2;
  a.volume = ctx->d_transvol;
  a.fuse_tile = (int)ctx->tune.fuse_z_tile;
  return a;
}

// Zero-padded product and inverse at M (k_spatial_pad.cu) on the spectra the
// unpadded forward left in d_spec (both sides); argmax into d_argmax[1].
static int run_spatial_padded(phgpu_ctx* ctx, const SpatialArgs& a, cudaStream_t st) {
  const int N = ctx->N, M = ctx->M;
  const size_t plane = (size_t)N * N * spatial_h2p(N);
  const int nch = a.laplace ? a.n_data_ch : (a.lowpass ? 2 : 1);
  {
    ProfScope ps(ctx, st, PS_FUSE_Z);
    for (int side = 0; side < 2; ++side)
      CK(launch_pad_zfft(a.spec + (size_t)side * a.n_data_ch * plane, plane, nch, N, N, N / 2 + 1, 0, ctx->plan_sp,
                         st));
    CK(cudaMemsetAsync(ctx->d_cspec_pad, 0, sizeof(float2) * (size_t)M * M * spatial_h2p(M), st));
    PadArgs pa;
    pa.N = N;
    pa.M = M;
    pa.pad = ctx->pad;
    pa.mode = a.laplace ? 1 : (a.lowpass ? 2 : 0);
    pa.n_ch = a.laplace ? a.n_total_ch : 1;
    pa.n_spec = a.laplace ? a.n_data_ch : 1;
    pa.spec_ch = a.n_data_ch;
    pa.first_ch = a.lowpass ? 1 : 0;
    pa.spec = a.spec;
    pa.prev_f = (a.laplace && ctx->prev_valid[0]) ? ctx->d_prev[0] : nullptr;
    pa.prev_g = (a.laplace && ctx->prev_valid[1]) ? ctx->d_prev[1] : nullptr;
    pa.x_natural_N = (spatial_slab_path(N) && a.plan_half) ? 1 : 0;
    pa.x_natural_M = ctx->has_pad_half ? 1 : 0;
    pa.planN = ctx->plan_sp;
    pa.planM = ctx->plan_pad;
    pa.bands = ctx->bands_sp;
    pa.lp_lo = a.lp_lo;
    pa.lp_hi = a.lp_hi;
    pa.inv_total = 1.0f / (float)a.n_total_ch;
    pa.cspec = ctx->d_cspec_pad;
    CK(launch_pad_fuse(pa, st));
    if (a.laplace) {
      // the buffers keep the last channel's shifted spectrum for the next call
      const int last = a.n_total_ch - 1;
      for (int side = 0; side < 2; ++side) {
        ctx->prev_valid[side] = last < a.n_data_ch;
        if (ctx->prev_valid[side])
          CK(cudaMemcpyAsync(ctx->d_prev[side], a.spec + (size_t)(side * a.n_data_ch + last) * plane,
                             sizeof(float2) * plane, cudaMemcpyDeviceToDevice, st));
      }
    }
    CK(launch_pad_zfft(ctx->d_cspec_pad, 0, 1, M, M, M / 2 + 1, 1, ctx->plan_pad, st));
  }
  SpatialArgs am = a;
  am.N = M;
  am.cspec = ctx->d_cspec_pad;
  am.plan = &ctx->plan_pad;
  am.plan_half = ctx->has_pad_half ? &ctx->plan_pad_half : nullptr;
  am.argmax_limit = ctx->corr_size;
  CK(cudaMemsetAsync(ctx->d_argmax + 1, 0, sizeof(unsigned long long), st));
  {
    ProfScope ps(ctx, st, PS_SPATIAL_INV);
    CK(launch_spatial_inverse(am, st));
  }
  return PHGPU_OK;
}

int phgpu_run_spatial(phgpu_ctx* ctx, int n_data, int n_total, int laplace, int means, cudaStream_t st) {
  SpatialArgs a = spatial_args(ctx, n_data, n_total, laplace, means);
  {
    ProfScope ps(ctx, st, PS_SPATIAL_FWD);
    CK(launch_spatial_forward(a, 0, st));
    CK(launch_spatial_forward(a, 1, st));
  }
  if (ctx->pad) {
    CKV(run_spatial_padded(ctx, a, st));
    CK(cudaMemcpyAsync(ctx->h_argmax + 1, ctx->d_argmax + 1, 2 * sizeof(unsigned long long),
                       cudaMemcpyDeviceToHost, st));
    ctx->have_trans = true;
    return PHGPU_OK;
  }
  CK(cudaMemsetAsync(ctx->d_argmax + 1, 0, sizeof(unsigned long long), st));
  {
    ProfScope ps(ctx, st, PS_FUSE_Z);
    CK(launch_spatial_fuse_z(a, st));
  }
  {
    ProfScope ps(ctx, st, PS_SPATIAL_INV);
    CK(launch_spatial_inverse(a, st));
  }
  CK(cudaMemcpyAsync(ctx->h_argmax + 1, ctx->d_argmax + 1, 2 * sizeof(unsigned long long),
                     cudaMemcpyDeviceToHost, st));
  ctx->have_trans = true;
  return PHGPU_OK;
}

int phgpu_spatial_correlate(phgpu_ctx* ctx, const double* const* f, const double* const* g, uint32_t C) {
  if (!ctx || !f || !g || C < 1 || C > 4) {
    if (ctx) ctx->err = "phgpu_spatial_correlate: 1..4 channels required";
    return PHGPU_ERR_INVALID;
  }
  if (ctx->prm.spatial_fusion == PHGPU_FUSION_LOW_PASS && C < 2) {
    ctx->err = "the low-pass spatial correlation uses channel 1: at least 2 channels required";
    return PHGPU_ERR_INVALID;
  }
  cudaSetDevice(ctx->prm.device);
  const size_t nv = (size_t)ctx->N * ctx->N * ctx->N;
  const int laplace = ctx->prm.spatial_fusion == PHGPU_FUSION_LAPLACE ? 1 : 0;
  std::vector<float> tmp(nv);
  for (int side = 0; side < 2; ++side) {
    ctx->clean_planes[side] = 0;
    ctx->grids_live[side] = false;
    const double* const* src = side == 0 ? f : g;
    for (uint32_t c = 0; c < C; ++c) {
      for (size_t i = 0; i < nv; ++i) tmp[i] = (float)src[c][i];
      CK(cudaMemcpy(ctx->d_grids[side] + c * nv, tmp.data(), sizeof(float) * nv, cudaMemcpyHostToDevice));
    }
  }
  CKV(phgpu_run_spatial(ctx, (int)C, (int)C, laplace, 1, ctx->s0));
  CK(cudaStreamSynchronize(ctx->s0));
  return PHGPU_OK;
}

int phgpu_spatial_correlate_voxelized(phgpu_ctx* ctx) {
  if (!ctx) return PHGPU_ERR_INVALID;
  if (!ctx->grids_live[0] || !ctx->grids_live[1] || ctx->vox_ch[0] != ctx->vox_ch[1]) {
    ctx->err = "both sides must be voxelised (phgpu_voxelize) with the same channel count first";
    return PHGPU_ERR_STATE;
  }
  cudaSetDevice(ctx->prm.device);
  const int laplace = ctx->prm.spatial_fusion == PHGPU_FUSION_LAPLACE ? 1 : 0;
  CKV(phgpu_run_spatial(ctx, ctx->vox_ch[0], (int)ctx->prm.n_channels, laplace, 0, ctx->s0));
  CK(cudaStreamSynchronize(ctx->s0));
  return PHGPU_OK;
}

int phgpu_spatial_result(phgpu_ctx* ctx, uint32_t* voxel, float* peak, double* corr_out) {
  if (!ctx) return PHGPU_ERR_INVALID;
  if (!ctx->have_trans) {
    ctx->err = "no spatial correlation computed";
    return PHGPU_ERR_STATE;
  }
  cudaSetDevice(ctx->prm.device);
  CK(cudaStreamSynchronize(ctx->s0));
  if (ctx->h_argmax[2] & 1ull) {
    ctx->err = "a bulk-copy wait in the translation kernels timed out";
    return PHGPU_ERR_CUDA;
  }
  const unsigned long long k = ctx->h_argmax[1];
  if (voxel) *voxel = unpack_index(k);
  if (peak) *peak = float_from_order_bits((uint32_t)(k >> 32));
  if (corr_out) {
    if (!ctx->d_transvol) {
      ctx->err = "volumes not kept (PHGPU_FLAG_KEEP_VOLUMES)";
      return PHGPU_ERR_STATE;
    }
    const size_t n = ctx->corr_size;  // N^3, or the reference's padded correlation length
    std::vector<float> tmp(n);
    CK(cudaMemcpy(tmp.data(), ctx->d_transvol, sizeof(float) * n, cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < n; ++i) corr_out[i] = tmp[i];
  }
  return PHGPU_OK;
}

// ------------------------------------------------------------------ pipeline

PairPlan pair_plan(const phgpu_ctx* ctx, bool t_refl, bool t_amb, bool s_refl, bool s_amb) {
  PairPlan pp;
  pp.laplace_s2 = ctx->prm.spherical_fusion == PHGPU_FUSION_LAPLACE ? 1 : 0;
  pp.laplace_sp = ctx->prm.spatial_fusion == PHGPU_FUSION_LAPLACE ? 1 : 0;
  pp.nd_s2 = std::max(t_amb ? 4 : (t_refl ? 3 : 2), s_amb ? 4 : (s_refl ? 3 : 2));
  pp.nd_sp = sp_channels(t_refl || s_refl, t_amb || s_amb);
  return pp;
}

int phgpu_pair_front(phgpu_ctx* ctx, const PairPlan& pp, bool until_phi) {
  // serialised profiling: the target's translation side on s0 as well, so the
  // per-stage events do not overlap
  cudaStream_t s0 = ctx->s0, s1 = ctx->prof_serial ? ctx->s0 : ctx->s1;
  // target translation side overlaps the rotation stage
  CK(cudaEventRecord(ctx->ev_a, s0));
  CK(cudaStreamWaitEvent(s1, ctx->ev_a, 0));
  CKV(phgpu_run_voxelize(ctx, 0, nullptr, pp.nd_sp, s1));
  const SpatialArgs sa = spatial_args(ctx, pp.nd_sp, (int)ctx->prm.n_channels, pp.laplace_sp, 0);
  {
    ProfScope ps(ctx, s1, PS_SPATIAL_FWD);
    CK(launch_spatial_forward(sa, 0, s1));
  }
  CKV(clear_voxelized(ctx, 0, s1));
  CK(cudaEventRecord(ctx->ev_b, s1));
  // rotation up to the fused spectra
  CKV(run_sample(ctx, 0, s0));
  CKV(run_sample(ctx, 1, s0));
  const bool mix = ctx->prm.spherical_fusion == PHGPU_FUSION_MIX;
  if (until_phi) {
    CKV(phgpu_run_sph_phi(ctx, pp.laplace_s2 ? pp.nd_s2 : 1, s0, mix));
  } else {
    CKV(phgpu_run_sph_front(ctx, pp.laplace_s2 ? pp.nd_s2 : 1, (int)ctx->prm.n_channels, pp.laplace_s2, s0, mix));
  }
  return PHGPU_OK;
}

int phgpu_pair_back(phgpu_ctx* ctx, const PairPlan& pp, const float* T, const float* T_dev) {
  cudaStream_t s0 = ctx->s0;
  const SpatialArgs sa = spatial_args(ctx, pp.nd_sp, (int)ctx->prm.n_channels, pp.laplace_sp, 0);
  CKV(phgpu_run_voxelize(ctx, 1, T, pp.nd_sp, s0, T_dev));
  {
    ProfScope ps(ctx, s0, PS_SPATIAL_FWD);
    CK(launch_spatial_forward(sa, 1, s0));
  }
  CKV(clear_voxelized(ctx, 1, s0));
  CK(cudaStreamWaitEvent(s0, ctx->ev_b, 0));
  if (ctx->pad) {
    CKV(run_spatial_padded(ctx, sa, s0));
  } else {
    CK(cudaMemsetAsync(ctx->d_argmax + 1, 0, sizeof(unsigned long long), s0));
    {
      ProfScope ps(ctx, s0, PS_FUSE_Z);
      CK(launch_spatial_fuse_z(sa, s0));
    }
    {
      ProfScope ps(ctx, s0, PS_SPATIAL_INV);
      CK(launch_spatial_inverse(sa, s0));
    }
  }
  // one read-back: rotation key, translation key, status (and the device transform)
  CK(cudaMemcpyAsync(ctx->h_argmax, ctx->d_argmax, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s0));
  if (T_dev) CK(cudaMemcpyAsync(ctx->h_T, T_dev, 12 * sizeof(float), cudaMemcpyDeviceToHost, s0));
  ctx->have_trans = true;
  return PHGPU_OK;
}

int phgpu_pair_finish(phgpu_ctx* ctx, const PairPlan& pp, bool device_pose, phgpu_pose* out) {
  cudaStream_t s0 = ctx->s0;
  if (ctx->h_argmax[2] & 2ull) {
    ctx->err = "a wait in the tensor-core SO(3) synthesis timed out";
    return PHGPU_ERR_CUDA;
  }
  float T[12];
  const unsigned long long rk = ctx->h_argmax[0];
  out->rot_bin = unpack_index(rk);
  out->rot_peak = float_from_order_bits((uint32_t)(rk >> 32));
  phgpu_pose_from_bin(out->rot_bin, (uint32_t)ctx->bw_out, out->zyz, out->quat, out->xyz, T);
  out->rot_omega[0] = out->rot_omega[1] = out->rot_omega[2] = 0.0;
  out->rot_omega[3] = 1.0;
  if (ctx->prm.rot_peak_neighbors > 0) {
    // Bingham fit over the linear-index window of the rotation volume: the
    // registration rotates the source by the mode (bingham-peak-based-eval.cc,
    // sph-opt-registration.cc:58-66)
    const uint32_t no = 2u * (uint32_t)ctx->bw_out;
    uint32_t first = 0, cnt = 0;
    phgpu_peak_window(out->rot_bin, no * no * no, ctx->prm.rot_peak_neighbors, &first, &cnt);
    std::vector<float> wf(cnt);
    CK(cudaMemcpy(wf.data(), ctx->d_rotvol + first, sizeof(float) * cnt, cudaMemcpyDeviceToHost));
    std::vector<double> w(wf.begin(), wf.end());
    if (phgpu_bingham_peak(w.data(), first, cnt, (uint32_t)ctx->bw_out, out->quat, out->rot_omega, out->xyz) !=
        PHGPU_OK) {
      ctx->err = "rotation peak neighbourhood has no positive weight";
      return PHGPU_ERR_STATE;
    }
    xyz_to_transform(out->xyz, T);
  }
  if (!device_pose || memcmp(T, ctx->h_T, sizeof(T)) != 0) {
    // translation with the host's transform: the host-pose cases, or a device
    // transform that differs in some bit from the host restatement (the two
    // sides' double trig functions may round differently)
    if (device_pose) ++ctx->pose_reruns;
    // the target's side finished with the registration; ev_b may last have
    // been recorded inside a captured graph (a server wave), which a stream
    // outside the graph cannot wait on: record it again on the idle stream
    CK(cudaEventRecord(ctx->ev_b, ctx->s1));
    CKV(phgpu_pair_back(ctx, pp, T, nullptr));
    CK(cudaStreamSynchronize(s0));
  }
  if (ctx->h_argmax[2] & 1ull) {
    ctx->err = "a bulk-copy wait in the translation kernels timed out";
    return PHGPU_ERR_CUDA;
  }
  const unsigned long long tk = ctx->h_argmax[1];
  out->voxel = unpack_index(tk);
  out->trans_peak = float_from_order_bits((uint32_t)(tk >> 32));
  // PhaseAligner::getNumberOfVoxels: N + 2 pad decodes the (padded) voxel
  const uint32_t N = (uint32_t)(ctx->pad ? ctx->M : ctx->N);
  const uint32_t xyz[3] = {(out->voxel / N) % N, out->voxel % N, out->voxel / (N * N)};
  for (int a = 0; a < 3; ++a)
    out->trans[a] = phgpu_translation_from_index((double)xyz[a], N, ctx->prm.spatial_discretize_lower,
                                                 ctx->prm.spatial_discretize_upper);
  for (int i = 0; i < 9; ++i) out->trans_cov[i] = 0.0;
  if (ctx->prm.trans_peak_neighbors > 0) {
    // Gaussian fit over the linear-index window of the translation volume:
    // the estimate is its mean (gaussian-peak-based-eval.cc, sph-opt-registration.cc:74-88)
    uint32_t first = 0, cnt = 0;
    phgpu_peak_window(out->voxel, ctx->corr_size, ctx->prm.trans_peak_neighbors, &first, &cnt);
    std::vector<float> wf(cnt);
    CK(cudaMemcpy(wf.data(), ctx->d_transvol + first, sizeof(float) * cnt, cudaMemcpyDeviceToHost));
    std::vector<double> w(wf.begin(), wf.end());
    if (phgpu_gaussian_peak(w.data(), first, cnt, N, ctx->prm.spatial_discretize_lower,
                            ctx->prm.spatial_discretize_upper, out->trans, out->trans_cov) != PHGPU_OK) {
      ctx->err = "translation peak neighbourhood has no positive weight sum";
      return PHGPU_ERR_STATE;
    }
  }
  return PHGPU_OK;
}

bool pair_device_pose(const phgpu_ctx* ctx) { return ctx->prm.rot_peak_neighbors == 0 && ctx->pad == 0; }

int phgpu_register_pair(phgpu_ctx* ctx, const phgpu_cloud* target, const phgpu_cloud* source,
                        phgpu_pose* out) {
  if (!ctx || !target || !source || !out) return PHGPU_ERR_INVALID;
  cudaSetDevice(ctx->prm.device);
  cudaStream_t s0 = ctx->s0;
  {
    ProfScope ps(ctx, s0, PS_UPLOAD);
    CKV(phgpu_upload_cloud(ctx, target, 0, s0));
    CKV(phgpu_upload_cloud(ctx, source, 1, s0));
  }
  const PairPlan pp = pair_plan(ctx, target->reflectivity, target->ambient, source->reflectivity, source->ambient);
  CKV(phgpu_pair_front(ctx, pp));
  So3Table t = so3_table(ctx);
  CKV(phgpu_run_so3_batch(&ctx, 1, t.table ? &t : nullptr, s0));
  // The rotation pose and the source's transform are computed on the device
  // and the translation follows without a host round trip.  A peak
  // neighbourhood fit (host, FP64) or the padded correlation (whose Laplace
  // mode carries state from one call to the next, so it cannot be redone)
  // take the transform from the host instead.
  const bool device_pose = pair_device_pose(ctx);
  if (device_pose) {
    PoseBatch pb;
    memset(&pb, 0, sizeof(pb));
    pb.count = 1;
    pb.bw_out = (uint32_t)ctx->bw_out;
    pb.argmax[0] = ctx->d_argmax;
    pb.T[0] = ctx->d_T;
    CK(launch_pose(pb, s0));
    CKV(phgpu_pair_back(ctx, pp, nullptr, ctx->d_T));
  } else {
    CK(cudaMemcpyAsync(ctx->h_argmax, ctx->d_argmax, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s0));
  }
  CK(cudaStreamSynchronize(s0));
  return phgpu_pair_finish(ctx, pp, device_pose, out);
}
