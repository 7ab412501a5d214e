// Context state shared by the C ABI (capi.cu) and the request server
// (server.cu).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/phaser_gpu.h"
#include "kernels.h"

// Stages timed by the optional per-stage profiler (phgpu_profile_*).
enum ProfStage {
  PS_UPLOAD = 0,
  PS_SAMPLE,
  PS_SHT,
  PS_FUSE_S2,
  PS_SO3_SYNTH,
  PS_SO3_FFT,
  PS_VOXELIZE,
  PS_SPATIAL_FWD,
  PS_FUSE_Z,
  PS_SPATIAL_INV,
  PS_COUNT
};

struct ProfRec {
  int stage;
  cudaEvent_t a, b;
};

struct phgpu_ctx {
  phgpu_params prm;
  int bw = 0, bw_out = 0, N = 0;
  float max_sq = 0.0f;
  std::string err;
  cudaStream_t s0 = nullptr, s1 = nullptr;
  cudaEvent_t ev_a = nullptr, ev_b = nullptr;
  // plans and tables
  phgpu::FftPlan plan_s2, plan_so3, plan_sp, plan_sp_half;
  bool has_sp_half = false;
  float2* d_tw[4] = {nullptr, nullptr, nullptr, nullptr};
  phgpu::FusionBands bands_s2, bands_sp;
  float4* d_grid = nullptr;
  double* d_weights = nullptr;
  float* d_legendre = nullptr;
  float* d_legendre_tc = nullptr;  // tensor-core layout of the Legendre table (precision != FP32)
  float* d_edges = nullptr;
  // clouds
  uint32_t cap_points = 0;
  float4* d_xyzi[2] = {nullptr, nullptr};
  float* d_refl[2] = {nullptr, nullptr};
  float* d_amb[2] = {nullptr, nullptr};
  void* d_sample_scratch[2] = {nullptr, nullptr};
  uint32_t* d_lin[2] = {nullptr, nullptr};
  uint32_t np[2] = {0, 0};
  int has_refl[2] = {0, 0}, has_amb[2] = {0, 0};
  // rotation
  float* d_samples = nullptr;  // [2][4][4B^2]
  float* d_mix = nullptr;      // [2][4B^2] single signal of PHGPU_FUSION_MIX
  int32_t* d_nn[2] = {nullptr, nullptr};
  float2* d_fphi = nullptr;  // SHT scratch: F_m(theta_k) per signal
  float2* d_coef = nullptr;
  float2* d_fused = nullptr;
  float2* d_S = nullptr;
  double* d_beta_tab = nullptr;  // [3][2 bw_out] for the Wigner seeds
  double* d_wig_tab = nullptr;   // Wigner recurrence tables (so3_wigner_table)
  float* d_wtable = nullptr;     // Wigner-d values of the tensor-core synthesis (precision != FP32)
  bool own_wigner_table = true;  // false: a server executor's slot (the executor holds the table)
  size_t* d_class_off = nullptr; // per-class offsets into d_wtable
  float* d_rotvol = nullptr;
  // translation
  float* d_grids[2] = {nullptr, nullptr};  // [(C+1)][N^3]
  uint8_t* d_rowlive[2] = {nullptr, nullptr};  // [N][N] rows holding a point of the last voxelisation
  uint8_t* d_slab_nz = nullptr;                 // [8][N] spectrum slabs that may be non-zero (k_slab_fwd)
  // leading grid planes (and row flags) known to be zero: a voxelisation whose
  // grids were cleared afterwards leaves them zero, so the next one needs no memset
  int clean_planes[2] = {0, 0};
  bool grids_live[2] = {false, false};  // grids hold the last voxelisation (not yet cleared)
  float2* d_spec = nullptr;
  float2* d_cspec = nullptr;
  float* d_transvol = nullptr;
  // zero-padded translation (spatial_zero_padding > 0): M = N + 2 pad
  int pad = 0, M = 0;
  uint32_t corr_size = 0;  // the reference's correlation length uint32(N^3 (M / N)^3) (M^3 or M^3 - 1)
  phgpu::FftPlan plan_pad, plan_pad_half;
  bool has_pad_half = false;
  float2* d_tw_pad[2] = {nullptr, nullptr};
  float2* d_cspec_pad = nullptr;           // [M][M][H2p(M)]
  float2* d_prev[2] = {nullptr, nullptr};  // Laplace: last channel spectrum of the previous call, per side
  bool prev_valid[2] = {false, false};
  int vox_ch[2] = {0, 0};
  // results
  unsigned long long* d_argmax = nullptr;  // [rot, trans]
  unsigned long long* h_argmax = nullptr;  // pinned
  float* d_T = nullptr;                    // [12] source transform of the device pose kernel
  float* h_T = nullptr;                    // pinned copy of d_T
  unsigned long long pose_reruns = 0;      // translations redone with the host transform
  phgpu_tuning tune{};                     // launch parameters (0 = built-in defaults)
  // point counts read by the kernels from device memory (the server's waves,
  // whose captured graphs take any count up to the capacity)
  bool dev_counts = false;
  uint32_t* d_np = nullptr;  // [2]
  uint32_t* h_np = nullptr;  // [2] pinned
  bool sampled[2] = {false, false};
  bool voxelized[2] = {false, false};
  bool have_rot = false, have_trans = false;
  // profiler
  bool prof_on = false;
  bool prof_serial = false;  // profiling with both halves of a registration on one stream
  std::vector<ProfRec> prof_recs;
  std::vector<cudaEvent_t> ev_pool;
  double prof_ms[PS_COUNT] = {0};
  unsigned long long prof_n[PS_COUNT] = {0};
  // bookkeeping
  std::vector<void*> allocs;
  size_t device_bytes = 0;
};

// Records start/end events of one stage on its stream when profiling is on.
struct ProfScope {
  phgpu_ctx* c;
  cudaStream_t s;
  int stage;
  cudaEvent_t a = nullptr;
  ProfScope(phgpu_ctx* ctx, cudaStream_t st, int stg);
  ~ProfScope();
};

int phgpu_ctx_init(phgpu_ctx* ctx);
// phgpu_ctx_create; wigner_table false leaves the tensor-core Wigner-d table
// to the caller (a server executor shares one among its slots)
int phgpu_ctx_create_internal(const phgpu_params* prm, phgpu_ctx** out, bool wigner_table);
int phgpu_upload_cloud(phgpu_ctx* ctx, const phgpu_cloud* c, int side, cudaStream_t st);
int phgpu_run_sph(phgpu_ctx* ctx, int n_data, int n_total, int laplace, cudaStream_t st, bool mix = false);
int phgpu_run_voxelize(phgpu_ctx* ctx, int side, const float* T12, int n_data, cudaStream_t st,
                       const float* T_dev = nullptr);
int phgpu_run_spatial(phgpu_ctx* ctx, int n_data, int n_total, int laplace, int means, cudaStream_t st);
phgpu::So3Args so3_args(phgpu_ctx* ctx);
int phgpu_run_sph_front(phgpu_ctx* ctx, int n_data, int n_total, int laplace, cudaStream_t st, bool mix = false);
int phgpu_run_so3_batch(phgpu_ctx* const* ctx, int k, const phgpu::So3Table* table, cudaStream_t st);

// One registration split for the server's waves: the front half on the
// context's streams (target translation side on s1, sampling + SHT + fusion
// on s0), the SO(3) stage (phgpu_run_so3_batch, batched across a wave), the
// pose kernel, the back half on s0 (source translation with the device or a
// host transform, one read-back into h_argmax / h_T) and the host finish
// (pose from the bin, transform check, peak neighbourhoods).
struct PairPlan {
  int nd_s2, nd_sp, laplace_s2, laplace_sp;
};
PairPlan pair_plan(const phgpu_ctx* ctx, bool t_refl, bool t_amb, bool s_refl, bool s_amb);
int phgpu_pair_front(phgpu_ctx* ctx, const PairPlan& pp, bool until_phi = false);
int phgpu_run_sph_phi(phgpu_ctx* ctx, int n_data, cudaStream_t st, bool mix);
int phgpu_run_sph_leg_fuse_batch(phgpu_ctx* const* ctx, int k, int n_data, int n_total, int laplace, bool mix,
                                 cudaStream_t st);
int phgpu_pair_back(phgpu_ctx* ctx, const PairPlan& pp, const float* T, const float* T_dev);
int phgpu_pair_finish(phgpu_ctx* ctx, const PairPlan& pp, bool device_pose, phgpu_pose* out);
bool pair_device_pose(const phgpu_ctx* ctx);
phgpu::So3Table so3_table(phgpu_ctx* ctx);

namespace phgpu {
bool make_fft_plan(int n, FftPlan* p, float2** d_tw, std::string* err);
bool fft_plan_radices(int n, int order, FftPlan* p);
FusionBands make_bands(uint32_t n, int levels, float div);
}  // namespace phgpu
