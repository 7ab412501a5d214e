/*
 * phaser_gpu.h -- C ABI of the B200 (sm_100a) implementation of PHASER's
 * correspondence-free registration hot path.
 *
 * Every entry point returns PHGPU_OK (0) or a negative status; no exception or
 * abort crosses the ABI.  A context owns one CUDA stream pair and all device
 * buffers for one (bandwidth, voxel grid) configuration; a context is not
 * thread-safe, distinct contexts may be used concurrently.  Array arguments
 * are host pointers unless the phgpu_cloud says otherwise.
 *
 * Each function names the reference interface it replaces (paths relative to
 * the ethz-asl/phaser tree).
 */
#ifndef PHASER_GPU_H_
#define PHASER_GPU_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PHGPU_OK 0
#define PHGPU_ERR_INVALID (-1)   /* bad argument or unsupported configuration */
#define PHGPU_ERR_CUDA (-2)      /* CUDA runtime error (message in phgpu_last_error) */
#define PHGPU_ERR_MEMORY (-3)    /* device allocation failed */
#define PHGPU_ERR_STATE (-4)     /* call out of order (e.g. result before correlate) */
#define PHGPU_ERR_LIMIT (-5)     /* size beyond a fixed limit (phgpu_sample_s2_noalloc) */

/* fusion modes */
#define PHGPU_FUSION_LAPLACE 0   /* SphericalCorrelationLaplace / SpatialCorrelationLaplace */
#define PHGPU_FUSION_NONE 1      /* SphericalCorrelation / SpatialCorrelation (channel 0) */
/* Low-pass variants: SphericalCorrelationLowPass (spherical-correlation-low-pass.cc:14-59)
 * correlates channel 0 keeping the B^2 coefficients whose FFT-shifted position
 * lies in [spherical_low_pass_lower, spherical_low_pass_upper); SpatialCorrelationLowPass
 * (spatial-correlation-low-pass.cc:40-90) correlates channel 1 keeping the
 * products whose FFT-shifted N^3 index has all three subscripts in
 * [spatial_low_pass_lower, min(spatial_low_pass_upper, N)]. */
#define PHGPU_FUSION_LOW_PASS 2
/* SphRegistration's single signal (spherical only; sph-registration.cc:166-198
 * with SphericalCorrelation::correlateSignals, spherical-correlation.cc:54-67,
 * 103-112): the sampled grids are mixed as 0.6 * intensity + 0.4 * range (in
 * double) and correlated as one channel without fusion.  Host sample arrays
 * (phgpu_sph_correlate, correlateSampledSignals) are taken as given: channel 0. */
#define PHGPU_FUSION_MIX 3

/* flags */
#define PHGPU_FLAG_KEEP_VOLUMES 1u /* also keep the full correlation volumes */

/* Arithmetic of the two contractions of the rotation path (the Legendre sums
 * of the forward SHT and the Wigner-d sums of the SO(3) synthesis):
 * FP32: CUDA-core FP32 sums (Legendre table from an FP64 recurrence once per
 * context; d-values from an FP64 recurrence run per call);
 * TF32X3 / BF16X3: tensor-core GEMMs over tables generated once per context
 * in FP64 and stored as FP32, each product split as hi*hi + hi*lo + lo*hi of
 * TF32 or BF16 parts with FP32 accumulation (bandwidth + spherical zero
 * padding <= 256).  Measured volume errors against FP64: FP32 <= 6e-7,
 * TF32X3 <= 2e-6, BF16X3 <= 1e-5 (its parts carry 16-17 bits). */
#define PHGPU_PRECISION_FP32 0
#define PHGPU_PRECISION_TF32X3 1
#define PHGPU_PRECISION_BF16X3 2

/* Configuration; names and defaults follow the reference's gflags
 * (phaser_common/src/common/core-gflags.cc:6-40,
 *  phaser_common/src/model/point-cloud.cc:19-20). */
typedef struct {
  uint32_t spherical_bandwidth;      /* phaser_core_spherical_bandwidth (75) */
  uint32_t spherical_zero_padding;   /* phaser_core_spherical_zero_padding (0) */
  uint32_t spatial_n_voxels;         /* phaser_core_spatial_n_voxels (100) */
  int32_t spatial_discretize_lower;  /* phaser_core_spatial_discretize_lower (-50) */
  int32_t spatial_discretize_upper;  /* phaser_core_spatial_discretize_upper (50) */
  uint32_t spatial_zero_padding;     /* phaser_core_spatial_zero_padding (0; N + 2 pad <= 1024) */
  float spatial_low_pass_lower;      /* phaser_core_spatial_low_pass_lower_bound (0) */
  float spatial_low_pass_upper;      /* phaser_core_spatial_low_pass_upper_bound (100000) */
  uint32_t n_channels;               /* channel count of the fusion (4) */
  uint32_t fusion_levels;            /* LaplacePyramid levels (5) */
  uint32_t spherical_fusion;         /* PHGPU_FUSION_* */
  uint32_t spatial_fusion;           /* PHGPU_FUSION_* */
  uint32_t max_points;               /* capacity per cloud (grows on demand) */
  uint32_t flags;                    /* PHGPU_FLAG_* */
  int32_t device;                    /* CUDA device ordinal */
  uint32_t rot_peak_neighbors;       /* bingham_peak_neighbors (0) */
  uint32_t trans_peak_neighbors;     /* gaussian_peak_neighbors (0) */
  uint32_t spherical_low_pass_lower; /* phaser_core_spherical_low_pass_lower_bound (0) */
  uint32_t spherical_low_pass_upper; /* phaser_core_spherical_low_pass_upper_bound (100000) */
  uint32_t precision;                /* PHGPU_PRECISION_* of the SO(3) synthesis (FP32) */
} phgpu_params;

/* A point cloud: x, y, z, intensity as float4 plus optional per-point
 * reflectivity and ambient values (phaser_common/include/phaser/model/
 * point-cloud.h:18-88).  on_device = 1 when the pointers are device memory. */
typedef struct {
  const float* xyzi;          /* 4 * n_points floats */
  const float* reflectivity;  /* n_points floats or NULL */
  const float* ambient;       /* n_points floats or NULL */
  uint32_t n_points;
  int32_t on_device;
} phgpu_cloud;

/* Registration result (phaser_core/src/backend/registration/
 * sph-opt-registration.cc:49-95). */
typedef struct {
  uint32_t rot_bin;     /* argmax of the SO(3) correlation, [beta][alpha][gamma] */
  float rot_peak;       /* |z|^2 at the bin */
  double zyz[3];        /* alpha, beta, gamma of the bin (rotation-utils.cc:197-208) */
  double quat[4];       /* w, x, y, z */
  double xyz[3];        /* Euler XYZ angles applied to the source (rotation-utils.cc:86-107) */
  uint32_t voxel;       /* argmax of the spatial correlation, [z][x][y] */
  float trans_peak;     /* correlation value at the voxel */
  double trans[3];      /* translation (translation-utils.cc:40-52) */
  double rot_omega[4];  /* normalised eigenvalues (ascending) of the peak's quaternion scatter matrix */
  double trans_cov[9];  /* covariance of the peak's translations (row-major) */
} phgpu_pose;

typedef struct phgpu_ctx phgpu_ctx;

/* Defaults of the reference's flags. */
int phgpu_params_default(phgpu_params* params);

/* Replaces the constructors SphericalCorrelation(bw, zero_padding)
 * (phaser_core/include/phaser/backend/correlation/spherical-correlation.h:19-21),
 * SpatialCorrelation(n_voxels, zero_padding) (spatial-correlation.h:15-17) and
 * PhaseAligner() (phase-aligner.cc:19-45): all tables, plans and buffers are
 * built once here and reused by every call. */
int phgpu_ctx_create(const phgpu_params* params, phgpu_ctx** out);
/* Replaces SphericalCorrelation::shutdown() (spherical-correlation.cc:31-52)
 * and the spatial destructors. */
int phgpu_ctx_destroy(phgpu_ctx* ctx);
/* Message of the last failing call on ctx (or of the last failing
 * phgpu_ctx_create when ctx is NULL). */
const char* phgpu_last_error(const phgpu_ctx* ctx);
/* The context's main CUDA stream (cudaStream_t). */
void* phgpu_stream(phgpu_ctx* ctx);

/* S^2 sampling of one cloud on the 2B x 2B grid: replaces
 * SphericalSampler::sampleUniformly (phaser_common/src/common/
 * spherical-sampler.cc:20-27).  side 0 = target (f), 1 = source (h). */
int phgpu_sample_s2(phgpu_ctx* ctx, const phgpu_cloud* cloud, int side);
/* Copies the sampled grids of a side to the host: n_channels x 4B^2 doubles
 * in the channel order {range, intensity, reflectivity, ambient}, and the
 * nearest-point index per grid direction (-1 when dropped).  Either may be NULL. */
int phgpu_get_samples(phgpu_ctx* ctx, int side, double* values, int32_t* nn_index);

/* S^2 sampling that allocates no device memory (no counterpart in the
 * reference; same kernels and results as phgpu_sample_s2 + phgpu_get_samples).
 * For callers that cannot allocate once running.  bw = params->spherical_
 * bandwidth, rejection radius from params->spatial_low_pass_* and
 * spatial_n_voxels as in a context.  The cloud must be on the device
 * (on_device = 1); values_dev receives 4 x 4bw^2 floats (channels {range,
 * intensity, reflectivity, ambient}, [theta][phi]) and nn_index_dev (or NULL)
 * 4bw^2 indices.  Runs asynchronously on `stream` (cudaStream_t, NULL = the
 * legacy default stream) on the current device.  Scratch is one fixed
 * device array per device: bw > PHGPU_NOALLOC_MAX_BANDWIDTH or n_points >
 * PHGPU_NOALLOC_MAX_POINTS returns PHGPU_ERR_LIMIT; calls that overlap on
 * one device race on the array.  The first call on each device looks the
 * array up (and may load the module there): make it before any stream
 * capture.  A call whose bandwidth differs from the previous call's on that
 * device also copies the grid directions into the array (host to device, on
 * `stream`, from pageable memory): make such a call outside stream capture
 * too (under capture it returns PHGPU_ERR_INVALID and enqueues nothing).
 * After cudaDeviceReset of a device, do not call this again in the same
 * process: the looked-up address belonged to the destroyed context. */
#define PHGPU_NOALLOC_MAX_POINTS (1 << 18)
#define PHGPU_NOALLOC_MAX_BANDWIDTH 128
int phgpu_sample_s2_noalloc(const phgpu_params* params, const phgpu_cloud* cloud, float* values_dev,
                            int32_t* nn_index_dev, void* stream);

/* SphericalCorrelationLaplace::correlateSampledSignals
 * (spherical-correlation-laplace.cc:14-40) / SphericalCorrelation::
 * correlateSampledSignals (spherical-correlation.cc:69-80): f[c], g[c] are
 * 4B^2 host doubles in [theta][phi] order. */
int phgpu_sph_correlate(phgpu_ctx* ctx, const double* const* f, const double* const* g,
                        uint32_t n_channels);
/* The same on the grids of the last phgpu_sample_s2 calls (no host copies). */
int phgpu_sph_correlate_sampled(phgpu_ctx* ctx);
/* Result of the last spherical correlation: the bin, its |z|^2 and, when
 * corr_out is not NULL (needs PHGPU_FLAG_KEEP_VOLUMES), the volume of
 * 8 bw_out^3 doubles: SphericalCorrelation::getCorrelation
 * (spherical-correlation.cc:114-116). */
int phgpu_sph_result(phgpu_ctx* ctx, uint32_t* bin, float* peak, double* corr_out);
/* SphericalCorrelation::getBandwidth (spherical-correlation.cc:118-120). */
uint32_t phgpu_sph_bandwidth(const phgpu_ctx* ctx);

/* PhaseAligner::discretizePointcloud (phase-aligner.cc:71-125) of one cloud,
 * optionally after the float 3x4 transform T (row-major) that
 * RotationUtils::RotateAroundXYZ applies (rotation-utils.cc:17-24). */
int phgpu_voxelize(phgpu_ctx* ctx, const phgpu_cloud* cloud, int side, const float* T12);
/* Per-point linear voxel index of the last voxelize of a side
 * (0xffffffff when skipped by the reference's guard). */
int phgpu_get_voxel_index(phgpu_ctx* ctx, int side, uint32_t* lin, uint32_t n_points);
/* SpatialCorrelationLaplace::correlateSignals / SpatialCorrelation::
 * correlateSignals (spatial-correlation-laplace.cc:17-51,
 * spatial-correlation.cc:128-175): f[c], g[c] are N^3 host doubles. */
int phgpu_spatial_correlate(phgpu_ctx* ctx, const double* const* f, const double* const* g,
                            uint32_t n_channels);
/* The same on the grids of the last phgpu_voxelize calls. */
int phgpu_spatial_correlate_voxelized(phgpu_ctx* ctx);
/* Result of the last spatial correlation: voxel, value and optionally the
 * correlation (PhaseAligner::getCorrelation, phase-aligner.cc:133-135) of
 * phgpu_spatial_correlation_size entries.  With spatial_zero_padding p the
 * correlation lives on M = N + 2p voxels per axis (the voxel decodes with M,
 * PhaseAligner::getNumberOfVoxels, phase-aligner.cc:137-139), and, as in the
 * reference, its value depends on the context's previous correlation in the
 * Laplace mode (the first channel reads the tail the previous call's last
 * channel left in the shifted buffer); the low-pass mode reproduces the
 * first call on a fresh reference object. */
int phgpu_spatial_result(phgpu_ctx* ctx, uint32_t* voxel, float* peak, double* corr_out);
/* SpatialCorrelation::getCorrelationSize (spatial-correlation.cc:219-221):
 * N^3, or uint32(N^3 ((N + 2p) / N)^3) in double with padding p (which is
 * (N + 2p)^3 - 1 for many N, p: the last voxel is then left out). */
uint32_t phgpu_spatial_correlation_size(const phgpu_ctx* ctx);

/* SphOptRegistration::registerPointCloud (sph-opt-registration.cc:34-47):
 * rotation, then translation of the rotated source.  The rotation pose and the
 * source's transform are computed on the device, so the pair runs as one
 * asynchronous chain with a single read-back; the host then recomputes the
 * transform from the bin and, should any bit differ (the two sides' double
 * trig functions may round differently), redoes the translation with the
 * host's transform.  With rot_peak_neighbors > 0 or spatial zero padding the
 * transform comes from the host. */
int phgpu_register_pair(phgpu_ctx* ctx, const phgpu_cloud* target, const phgpu_cloud* source,
                        phgpu_pose* out);
/* Translations phgpu_register_pair redid with the host transform on ctx. */
unsigned long long phgpu_pose_reruns(const phgpu_ctx* ctx);

/* Host pose arithmetic of the reference (rotation-utils.cc:86-143, 197-208;
 * translation-utils.cc:40-52). */
int phgpu_pose_from_bin(uint32_t bin, uint32_t bw_out, double* zyz, double* quat, double* xyz,
                        float* T12);
/* Peak-neighbourhood statistics (host; the registration calls them when
 * rot/trans_peak_neighbors > 0 with the volume values of the linear-index
 * window around the argmax).
 *
 * BinghamPeakBasedEval::fitRotationalBinghamDistribution
 * (phaser_core/src/backend/uncertainty/bingham-peak-based-eval.cc:22-91) with
 * Bingham::fit / fitToMoment (phaser_common/src/distribution/bingham.cc:239-295):
 * values[i] weights the quaternion of SO(3) bin first_bin + i (normalised to
 * sum 1 when count > 1); the scatter matrix sum_i w_i q_i q_i^T is
 * eigen-decomposed; mode4 (w, x, y, z, w >= 0) is its principal eigenvector --
 * the mode the reference's estimate returns -- and omega4 its eigenvalues in
 * ascending order divided by their sum.  xyz3 gets the Euler angles of the
 * mode (rotation-utils.cc:86-93).  The concentrations, which the reference
 * fits with an external optimiser, are not computed.
 *
 * GaussianPeakBasedEval::fitTranslationalNormalDist (gaussian-peak-based-eval.cc:
 * 42-101) with Gaussian::setMeanAndCov (phaser_common/src/distribution/
 * gaussian.cc:47-55): values[i] (normalised to sum 1) weights the translation
 * of voxel first_voxel + i; mean3 and cov9 (row-major) are the weighted mean
 * and covariance. */
int phgpu_bingham_peak(const double* values, uint32_t first_bin, uint32_t count, uint32_t bw_out,
                       double* mode4, double* omega4, double* xyz3);
int phgpu_gaussian_peak(const double* values, uint32_t first_voxel, uint32_t count, uint32_t n_voxels,
                        int32_t lower, int32_t upper, double* mean3, double* cov9);
/* Smoothed z-score peak extraction of a correlation vector
 * (ZScorePeakExtraction::extractPeaks / calculateSmoothedZScore,
 * phaser_core/src/backend/uncertainty/z-score-peak-extraction.cc:42-112), on
 * the host in FP64: lag = min(lag_max, (uint32)(n * lag_percentile)); the
 * mean and sample standard deviation of a window of `lag` values slide along
 * the vector, and an index i > lag whose value exceeds filter_threshold and
 * lies more than threshold deviations from the window mean is a peak when it
 * lies above the mean; such a value is damped (influence * x + (1 - influence)
 * * previous) before the window moves on.  Peaks are written in ascending
 * order; *n_peaks receives their count (PHGPU_ERR_LIMIT when it exceeds
 * capacity, the first `capacity` written).  Parameter checks as the
 * reference's constructor: 0 < lag_percentile < 1, threshold > 0,
 * 0 <= influence <= 1. */
typedef struct phgpu_zscore_params {
  double lag_percentile;    /* z_score_lag_percentile (0.05) */
  uint32_t lag_max;         /* z_score_lag_max (20) */
  double threshold;         /* z_score_threshold (4.33) */
  double influence;         /* z_score_influence (0.05) */
  double filter_threshold;  /* z_score_filter_threshold (0.405) */
} phgpu_zscore_params;
int phgpu_zscore_params_default(phgpu_zscore_params* params);
int phgpu_zscore_peaks(const double* values, uint64_t n, const phgpu_zscore_params* params, uint32_t* peaks,
                       uint64_t capacity, uint64_t* n_peaks);

/* The linear-index window [first, first + count) the two evaluators take
 * around an argmax `index` of an n-element volume for k neighbours
 * (calculateStartEndNeighbor, gaussian-peak-based-eval.cc:31-41). */
void phgpu_peak_window(uint32_t index, uint32_t n, uint32_t k, uint32_t* first, uint32_t* count);

double phgpu_translation_from_index(double index, uint32_t n_voxels, int32_t lower,
                                    int32_t upper);

/* ------------------------------------------------------------------ tuning
 * Launch parameters chosen per shape by the project's autotuner (no reference
 * counterpart: the reference plans its FFTs with FFTW_ESTIMATE on every call,
 * spherical-correlation.cc:122-206).  0 selects the built-in default.  Every
 * value gives the same results except radix_order, which reorders the stages
 * of runtime FFT plans (lengths other than 64, 128, 200, 256, 320 and 512) and
 * so their FP32 rounding. */
typedef struct {
  uint32_t fuse_z_tile;    /* ky columns per block of the translation z pass: 2, 4, 8, 16 */
  uint32_t so3_beta_tile;  /* betas per block of the SO(3) alpha transform: 8, 16, 32 */
  uint32_t tc_chunk;       /* degrees per chunk of the tensor-core synthesis: 16, 32 */
  uint32_t radix_order;    /* runtime FFT plans: 0 radix 8 first, 1 radix 4 first, 2 odd radices first */
} phgpu_tuning;
int phgpu_tuning_get(const phgpu_ctx* ctx, phgpu_tuning* out);
/* PHGPU_ERR_INVALID for a value the context's shape cannot take. */
int phgpu_tuning_set(phgpu_ctx* ctx, const phgpu_tuning* t);
/* Coordinate search: the candidates of each parameter in turn, each timed on
 * `reps` registrations of the given pair (after one warm-up) with this
 * context's buffers by the per-stage CUDA events of the stage the parameter
 * affects (the whole registration for the radix order).  Keeps the fastest on
 * ctx and returns it with the registration's device time in ms (sum of the
 * stage events) under it. */
int phgpu_autotune(phgpu_ctx* ctx, const phgpu_cloud* target, const phgpu_cloud* source, uint32_t reps,
                   phgpu_tuning* best, double* ms_per_pair);

/* ------------------------------------------------------------------ tracing
 * Per-stage device time measured with CUDA events on each stage's launching
 * stream (the reference times stages on the host clock,
 * phaser_common/include/phaser/common/statistic-utils.h:10-18). */
/* enable 1: events on each stage's own stream (the two clouds' stages of a
 * registration overlap, and so do their events); 2: the registration's two
 * streams serialised on one, so every stage's events time it alone. */
int phgpu_profile_enable(phgpu_ctx* ctx, int enable);
/* Accumulated milliseconds and call counts per stage since the last read
 * (synchronises the context's streams; resets the accumulators). */
int phgpu_profile_read(phgpu_ctx* ctx, double* ms, unsigned long long* calls, int n);
int phgpu_profile_stage_count(void);
const char* phgpu_profile_stage_name(int stage);
/* Kernels launched by this library since it was loaded (all contexts). */
unsigned long long phgpu_launch_count(void);

/* ------------------------------------------------------------------ ingest
 * PLY reading (replaces data::PlyHelper::readPlyFromFile +
 * PointCloud::parsePlyPointCloud, phaser_common/src/common/data/
 * ply-helper.cc:26-64, phaser_common/src/model/point-cloud.cc:313-348).
 * field_names: the intensity, reflectivity, ambient and range property names
 * (the reference's --phaser_ply_*_str flags); NULL, or a NULL entry, selects
 * the defaults "intensity", "reflectivity", "noise", "range".  x, y, z and
 * intensity are required (PHGPU_ERR_INVALID otherwise, where the reference
 * aborts).  Host only; the outputs are typically pinned for the upload. */
#define PHGPU_PLY_REFLECTIVITY 1u
#define PHGPU_PLY_AMBIENT 2u
#define PHGPU_PLY_RANGE 4u
/* Vertex count and which optional fields exist (PHGPU_PLY_* bits). */
int phgpu_ply_info(const char* path, const char* const* field_names, uint32_t* n_points, uint32_t* present);
/* x, y, z, intensity into xyzi (4 floats per point); the optional fields into
 * their arrays when non-NULL and present (left untouched when absent).
 * PHGPU_ERR_LIMIT when the file holds more than `capacity` vertices. */
int phgpu_ply_read(const char* path, const char* const* field_names, float* xyzi, float* reflectivity,
                   float* ambient, float* range, uint32_t capacity, uint32_t* n_points);
/* Message of the last failed phgpu_ply_* call on this thread. */
const char* phgpu_ply_last_error(void);

/* Voxel-grid downsampling on the GPU (replaces preproc::VoxelGridCmd,
 * phaser_pre/src/commands/voxel-grid-cmd.cc:11-22, i.e. pcl::VoxelGrid with
 * downsample_all_data on PointXYZI).  Each occupied leaf of the grid
 * anchored at floor(min / leaf) becomes one point, the float mean of x, y, z
 * and intensity of its points; leaves come out in increasing leaf index
 * (x fastest, then y, then z) and points inside a leaf are summed in input
 * order.  Points with a non-finite coordinate are dropped.  When the leaf
 * count would overflow int32 the input is returned unchanged (as the
 * reference does).  Reflectivity and ambient, when given, are averaged over the
 * same leaves (the reference leaves them unfiltered). */
typedef struct phgpu_voxel_grid phgpu_voxel_grid;
int phgpu_voxel_grid_create(uint32_t max_points, int32_t device, phgpu_voxel_grid** out);
int phgpu_voxel_grid_destroy(phgpu_voxel_grid* vg);
/* leaf: x, y, z leaf sizes (> 0); min_points_per_voxel: leaves with fewer
 * points are dropped (pcl::VoxelGrid::setMinimumPointsNumberPerVoxel, 0 by
 * default).  The outputs hold in->n_points entries at least; out_on_device
 * says whether they are device (1) or host (0) memory.  Synchronises the
 * filter's stream before returning *n_out. */
int phgpu_voxel_grid_filter(phgpu_voxel_grid* vg, const phgpu_cloud* in, const float leaf[3],
                            uint32_t min_points_per_voxel, float* out_xyzi, float* out_reflectivity,
                            float* out_ambient, int out_on_device, uint32_t* n_out);
const char* phgpu_voxel_grid_last_error(const phgpu_voxel_grid* vg);

/* ------------------------------------------------------------------ serving
 * Continuous-batching request server (no reference counterpart: the
 * reference registers one pair at a time, sph-opt-registration.cc:34-47).
 * Requests are grouped by shape (bandwidth, voxel grid, fusion, precision and
 * the clouds' optional channels) into waves of up to max_wave pairs; a wave is
 * one CUDA graph launch over device-resident per-slot state, with each SO(3)
 * stage batched across the wave (the tensor-core synthesis reads the shape's
 * Wigner-d table once per wave).  `lanes` waves run concurrently, so requests
 * that arrive while one wave is on the GPU join the next.  Executors (the
 * per-shape slot sets) are admitted against the HBM budget; idle ones are
 * evicted, least recently used first, when a new shape needs the memory. */
typedef struct phgpu_server phgpu_server;

typedef struct {
  uint64_t hbm_budget_bytes;   /* admission budget (150 GB when 0) */
  uint32_t max_wave;           /* pairs per wave (16 when 0; at most 32) */
  uint32_t max_points;         /* capacity per cloud (2^18 when 0); larger clouds are refused */
  int32_t device;
  uint32_t flags;              /* PHGPU_SERVER_* */
  uint32_t lanes;              /* waves in flight at once (2 when 0) */
  uint32_t max_delay_us;       /* longest a request is held back to fill a wave while another wave
                                  runs (500 when 0); an idle GPU starts a wave at once */
} phgpu_server_params;

/* Host clouds are read in place by the worker (copied to the device inside the
 * wave, asynchronously when the memory is pinned) instead of being copied at
 * submit; the caller keeps them valid until the ticket completes. */
#define PHGPU_SERVER_BORROW_HOST 1u

typedef struct {
  uint64_t waves;           /* waves run */
  uint64_t requests;        /* requests completed in waves */
  uint64_t graph_captures;  /* CUDA graphs captured (one per executor and wave size) */
  uint64_t direct_waves;    /* waves launched without a graph (their capture was invalidated by other
                               CUDA work of the process that synchronised the device) */
  uint64_t evictions;       /* executors evicted to admit another shape */
  uint64_t pose_reruns;     /* translations redone with the host transform */
  uint64_t executors;       /* executors resident now */
  uint64_t bytes_in_use;    /* device bytes of the resident executors */
} phgpu_server_stats;

int phgpu_server_create(const phgpu_server_params* params, phgpu_server** out);
int phgpu_server_destroy(phgpu_server* srv);
/* Submits one pair; params gives the shape (bandwidth, voxels, bounds,
 * precision).  Host clouds are copied before the call returns (unless
 * PHGPU_SERVER_BORROW_HOST); device clouds (on_device = 1 for both) are read in
 * place and must stay valid until the ticket completes.  Spatial zero padding
 * is refused (PHGPU_ERR_INVALID), clouds above max_points too (PHGPU_ERR_LIMIT).
 * *ticket identifies the request. */
int phgpu_server_submit(phgpu_server* srv, const phgpu_params* params, const phgpu_cloud* target,
                        const phgpu_cloud* source, uint64_t* ticket);
/* Non-blocking: 1 and the pose when the ticket finished, 0 otherwise. */
int phgpu_server_poll(phgpu_server* srv, uint64_t ticket, phgpu_pose* out, double* latency_ms);
/* The same, also copying the request's correlation volumes ((2 bw_out)^3 and
 * N^3 floats, layouts as phgpu_sph_result / phgpu_spatial_result) when it was
 * submitted with PHGPU_FLAG_KEEP_VOLUMES; either pointer may be NULL. */
int phgpu_server_poll_volumes(phgpu_server* srv, uint64_t ticket, phgpu_pose* out, double* latency_ms,
                              float* rot_volume, float* trans_volume);
/* Blocks until every submitted request finished. */
int phgpu_server_drain(phgpu_server* srv);
int phgpu_server_get_stats(phgpu_server* srv, phgpu_server_stats* out);
/* Tuning the server applies to executors created afterwards for the shape of
 * `shape` (bandwidth, spherical zero padding, voxels, precision). */
int phgpu_server_set_tuning(phgpu_server* srv, const phgpu_params* shape, const phgpu_tuning* t);
const char* phgpu_server_last_error(const phgpu_server* srv);

#ifdef __cplusplus
}
#endif

#endif /* PHASER_GPU_H_ */
