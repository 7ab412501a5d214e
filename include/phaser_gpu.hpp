// phaser_gpu.hpp -- header-only C++ drop-ins for phaser_core's correlation and
// aligner classes, backed by the C ABI of phaser_gpu.h (B200, sm_100a).
//
// The class names, constructor arguments and member functions follow
//   SphericalCorrelation          phaser_core/include/phaser/backend/correlation/spherical-correlation.h:19-33
//   SphericalCorrelationLaplace   .../spherical-correlation-laplace.h
//   SpatialCorrelation            .../spatial-correlation.h:15-23
//   SpatialCorrelationLaplace     .../spatial-correlation-laplace.h
//   SphericalCorrelationLowPass   .../spherical-correlation-low-pass.h
//   SpatialCorrelationLowPass     .../spatial-correlation-low-pass.h
//   PhaseAligner                  phaser_core/include/phaser/backend/alignment/phase-aligner.h:17-26
//   SphOptRegistration            phaser_core/include/phaser/backend/registration/sph-opt-registration.h
//   SphericalSampler, FunctionValue
//                                 phaser_common/include/phaser/common/spherical-sampler.h,
//                                 phaser_common/include/phaser/model/function-value.h
//   PlyHelper, PlyPointCloud      phaser_common/include/phaser/common/data/ply-helper.h,
//                                 phaser_common/include/phaser/model/ply-point-cloud.h
//   VoxelGridCmd                  phaser_pre/include/phaser_pre/commands/voxel-grid-cmd.h
// so a caller swaps the include and the namespace (phaser_gpu instead of
// phaser_core).  Errors throw std::runtime_error (the reference aborts through
// glog CHECKs instead).  Eigen::VectorXd arguments are accepted when Eigen is
// included before this header (PHASER_GPU_WITH_EIGEN), raw double pointers
// otherwise.
#ifndef PHASER_GPU_HPP_
#define PHASER_GPU_HPP_

#include <cstdint>
#include <algorithm>
#include <memory>
#include <set>
#include <stdexcept>
#include <string>
#include <vector>

#include "phaser_gpu.h"

#if defined(EIGEN_WORLD_VERSION) && !defined(PHASER_GPU_WITH_EIGEN)
#define PHASER_GPU_WITH_EIGEN 1
#endif

namespace phaser_gpu {

using SampledSignal = std::vector<double>;

// Flag-backed parameters with the reference's defaults
// (phaser_common/src/common/core-gflags.cc:6-40).
inline phgpu_params default_params() {
  phgpu_params p;
  phgpu_params_default(&p);
  return p;
}

namespace detail {
inline void check(int rc, const phgpu_ctx* ctx, const char* what) {
  if (rc != PHGPU_OK)
    throw std::runtime_error(std::string(what) + ": " + phgpu_last_error(ctx));
}

// Owns one device context.
class Context {
 public:
  explicit Context(const phgpu_params& p) {
    check(phgpu_ctx_create(&p, &ctx_), nullptr, "phgpu_ctx_create");
  }
  ~Context() { phgpu_ctx_destroy(ctx_); }
  Context(const Context&) = delete;
  Context& operator=(const Context&) = delete;
  phgpu_ctx* get() const { return ctx_; }

 private:
  phgpu_ctx* ctx_ = nullptr;
};
}  // namespace detail

// One direction's sample (model::FunctionValue): the values of the nearest
// cloud point (the 1-NN sampler feeds each direction one point), 0 when the
// nearest point lies beyond the rejection radius (nn_index -1).
struct FunctionValue {
  double range = 0.0, intensity = 0.0, reflectivity = 0.0, ambient = 0.0;
  int32_t nn_index = -1;
  double getAveragedRange() const noexcept { return range; }
  double getAveragedIntensity() const noexcept { return intensity; }
  double getAveragedReflectivity() const noexcept { return reflectivity; }
  double getAveragedAmbientNoise() const noexcept { return ambient; }
};

// SphericalCorrelation(bw, zero_padding): single-signal correlation
// (correlateSampledSignals uses the first channel, spherical-correlation.cc:69-80).
class SphericalCorrelation {
 public:
  explicit SphericalCorrelation(const uint32_t bw = 100, const uint32_t zero_padding = 0,
                                const phgpu_params& base = default_params())
      : SphericalCorrelation(bw, zero_padding, PHGPU_FUSION_NONE, base) {}
  virtual ~SphericalCorrelation() { delete ctx_; }

  // f[c], g[c]: 4 bw^2 samples in [theta][phi] order.
  virtual void correlateSampledSignals(const std::vector<SampledSignal>& f,
                                       const std::vector<SampledSignal>& g) {
    if (f.size() != g.size() || f.empty())
      throw std::invalid_argument("correlateSampledSignals: channel counts differ or are zero");
    const size_t nc = fusion_ == PHGPU_FUSION_LAPLACE ? f.size() : 1;
    std::vector<const double*> fp(nc), gp(nc);
    for (size_t c = 0; c < nc; ++c) {
      if (f[c].size() != 4ull * bw_ * bw_ || g[c].size() != 4ull * bw_ * bw_)
        throw std::invalid_argument("correlateSampledSignals: expected 4 bw^2 samples per channel");
      fp[c] = f[c].data();
      gp[c] = g[c].data();
    }
    detail::check(phgpu_sph_correlate(ctx_->get(), fp.data(), gp.data(), (uint32_t)nc), ctx_->get(),
                  "phgpu_sph_correlate");
    have_ = true;
  }

  // SphericalCorrelation::correlateSignals (spherical-correlation.cc:54-67):
  // one signal per side, 0.6 * intensity + 0.4 * range of every direction
  // (retrieveInterpolation, :103-112), correlated by correlateSampledSignals
  // (virtual, as in the reference: the Laplace class refuses one channel).
  void correlateSignals(const std::vector<FunctionValue>& f1, const std::vector<FunctionValue>& f2) {
    SampledSignal a, b;
    retrieveInterpolation(f1, &a);
    retrieveInterpolation(f2, &b);
    correlateSampledSignals({a}, {b});
  }
  static void retrieveInterpolation(const std::vector<FunctionValue>& f, SampledSignal* out) {
    out->reserve(out->size() + f.size());
    for (const FunctionValue& v : f) out->push_back(0.6 * v.getAveragedIntensity() + 0.4 * v.getAveragedRange());
  }

  // |z|^2 over the (2 bw_out)^3 grid, [beta][alpha][gamma].
  std::vector<double> getCorrelation() const {
    std::vector<double> out((size_t)8 * bw_out_ * bw_out_ * bw_out_);
    if (have_)
      detail::check(phgpu_sph_result(ctx_->get(), nullptr, nullptr, out.data()), ctx_->get(),
                    "phgpu_sph_result");
    return out;
  }
  // argmax bin of the last correlation (what PhaseCorrelationEval extracts)
  uint32_t getPeakBin() const {
    uint32_t b = 0;
    detail::check(phgpu_sph_result(ctx_->get(), &b, nullptr, nullptr), ctx_->get(), "phgpu_sph_result");
    return b;
  }
  uint32_t getBandwidth() const noexcept { return bw_out_; }
  void shutdown() {}

 protected:
  SphericalCorrelation(const uint32_t bw, const uint32_t zero_padding, const uint32_t fusion,
                       const phgpu_params& base)
      : bw_(bw), bw_out_(bw + zero_padding), fusion_(fusion) {
    phgpu_params p = base;
    p.spherical_bandwidth = bw;
    p.spherical_zero_padding = zero_padding;
    p.spherical_fusion = fusion;
    p.flags |= PHGPU_FLAG_KEEP_VOLUMES;
    if (p.spatial_n_voxels == 0) p.spatial_n_voxels = 4;
    ctx_ = new detail::Context(p);
  }
  uint32_t bw_, bw_out_, fusion_;
  detail::Context* ctx_ = nullptr;
  bool have_ = false;
};

// SphericalCorrelationLaplace: channel fusion, >= 2 channels
// (spherical-correlation-laplace.cc:14-17).
class SphericalCorrelationLaplace : public SphericalCorrelation {
 public:
  explicit SphericalCorrelationLaplace(const uint32_t bw = 100, const uint32_t zero_padding = 0,
                                       const phgpu_params& base = default_params())
      : SphericalCorrelation(bw, zero_padding, PHGPU_FUSION_LAPLACE, base) {}
  void correlateSampledSignals(const std::vector<SampledSignal>& f,
                               const std::vector<SampledSignal>& g) override {
    if (f.size() < 2) throw std::invalid_argument("SphericalCorrelationLaplace needs at least 2 channels");
    SphericalCorrelation::correlateSampledSignals(f, g);
  }
};

// SphericalCorrelationLowPass(bw, zero_padding): channel 0 with the B^2
// coefficients outside the FFT-shifted band [lower, upper) removed
// (spherical-correlation-low-pass.cc:14-59); the band comes from
// base.spherical_low_pass_lower / _upper (the reference's flags).
class SphericalCorrelationLowPass : public SphericalCorrelation {
 public:
  explicit SphericalCorrelationLowPass(const uint32_t bw = 100, const uint32_t zero_padding = 0,
                                       const phgpu_params& base = default_params())
      : SphericalCorrelation(bw, zero_padding, PHGPU_FUSION_LOW_PASS, base) {}
};

// SpatialCorrelation(n_voxels, zero_padding) / SpatialCorrelationLaplace.
// correlateSignals returns a pointer owned by the object, valid until the next
// call, to getCorrelationSize() values (spatial-correlation.cc:163-206); with
// zero padding the correlation covers (n_voxels + 2 zero_padding)^3 voxels.
class SpatialCorrelation {
 public:
  explicit SpatialCorrelation(const uint32_t n_voxels, const uint32_t zero_padding = 0,
                              const phgpu_params& base = default_params())
      : n_(n_voxels), pad_(zero_padding) {
    make(base, PHGPU_FUSION_NONE);
  }
  virtual ~SpatialCorrelation() { delete ctx_; }

  double* correlateSignals(const std::vector<const double*>& f, const std::vector<const double*>& g) {
    if (f.size() != g.size() || f.empty())
      throw std::invalid_argument("correlateSignals: channel counts differ or are zero");
    detail::check(phgpu_spatial_correlate(ctx_->get(), f.data(), g.data(), (uint32_t)f.size()),
                  ctx_->get(), "phgpu_spatial_correlate");
    c_.resize(getCorrelationSize());
    detail::check(phgpu_spatial_result(ctx_->get(), &peak_voxel_, nullptr, c_.data()), ctx_->get(),
                  "phgpu_spatial_result");
    return c_.data();
  }
#ifdef PHASER_GPU_WITH_EIGEN
  double* correlateSignals(const std::vector<Eigen::VectorXd*>& f, const std::vector<Eigen::VectorXd*>& g) {
    std::vector<const double*> fp, gp;
    for (auto* v : f) fp.push_back(v->data());
    for (auto* v : g) gp.push_back(v->data());
    return correlateSignals(fp, gp);
  }
#endif
  uint32_t getZeroPadding() const { return pad_; }
  uint32_t getCorrelationSize() const { return phgpu_spatial_correlation_size(ctx_->get()); }
  uint32_t getPeakVoxel() const { return peak_voxel_; }

 protected:
  SpatialCorrelation(const uint32_t n_voxels, const uint32_t zero_padding, int fusion, const phgpu_params& base)
      : n_(n_voxels), pad_(zero_padding) {
    make(base, fusion);
  }
  void make(const phgpu_params& base, int fusion) {
    phgpu_params p = base;
    p.spatial_n_voxels = n_;
    p.spatial_zero_padding = pad_;
    p.spatial_fusion = (uint32_t)fusion;
    p.flags |= PHGPU_FLAG_KEEP_VOLUMES;
    if (p.spherical_bandwidth < 2) p.spherical_bandwidth = 2;
    ctx_ = new detail::Context(p);
  }
  uint32_t n_, pad_;
  detail::Context* ctx_ = nullptr;
  std::vector<double> c_;
  uint32_t peak_voxel_ = 0;
};

class SpatialCorrelationLaplace : public SpatialCorrelation {
 public:
  explicit SpatialCorrelationLaplace(const uint32_t n_voxels, const uint32_t zero_padding = 0,
                                     const phgpu_params& base = default_params())
      : SpatialCorrelation(n_voxels, zero_padding, PHGPU_FUSION_LAPLACE, base) {}
};

// SpatialCorrelationLowPass(n_voxels, zero_padding[, lower, upper]): channel 1
// of the signals, products kept inside the FFT-shifted cube [lower, upper]^3
// (spatial-correlation-low-pass.cc:11-98).  Without bounds: the reference's
// flags, upper clipped to n_voxels.
class SpatialCorrelationLowPass : public SpatialCorrelation {
 public:
  explicit SpatialCorrelationLowPass(const uint32_t n_voxels, const uint32_t zero_padding = 0,
                                     const phgpu_params& base = default_params())
      : SpatialCorrelationLowPass(n_voxels, zero_padding,
                                  base.spatial_low_pass_lower > 0.f ? (uint32_t)base.spatial_low_pass_lower : 0u,
                                  std::min<uint32_t>(base.spatial_low_pass_upper > 0.f
                                                         ? (uint32_t)base.spatial_low_pass_upper : 0u,
                                                     n_voxels),
                                  base) {}
  SpatialCorrelationLowPass(const uint32_t n_voxels, const uint32_t zero_padding, const uint32_t lower,
                            const uint32_t upper, const phgpu_params& base = default_params())
      : SpatialCorrelation(n_voxels, zero_padding, PHGPU_FUSION_LOW_PASS, with_bounds(base, lower, upper)),
        lower_(lower), upper_(upper) {}
  uint32_t getLowerBound() const noexcept { return lower_; }
  uint32_t getUpperBound() const noexcept { return upper_; }
  uint32_t getNumberOfIndices() const noexcept {
    const uint32_t w = upper_ >= lower_ ? upper_ - lower_ + 1 : 0;
    return w * w * w;
  }

 private:
  static phgpu_params with_bounds(phgpu_params p, uint32_t lower, uint32_t upper) {
    p.spatial_low_pass_lower = (float)lower;
    p.spatial_low_pass_upper = (float)upper;
    return p;
  }
  uint32_t lower_, upper_;
};

// A cloud as the aligner and registration see it: x, y, z, intensity per
// point and optional reflectivity / ambient (phaser_common's model::PointCloud).
struct CloudView {
  const float* xyzi = nullptr;
  const float* reflectivity = nullptr;
  const float* ambient = nullptr;
  uint32_t n_points = 0;
  bool on_device = false;
  phgpu_cloud c() const { return phgpu_cloud{xyzi, reflectivity, ambient, n_points, on_device ? 1 : 0}; }
};

// PhaseAligner: voxelise both clouds and correlate (phase-aligner.cc:47-69).
class PhaseAligner {
 public:
  explicit PhaseAligner(const phgpu_params& base = default_params()) : prm_(base) {
    phgpu_params p = base;
    p.flags |= PHGPU_FLAG_KEEP_VOLUMES;
    ctx_ = new detail::Context(p);
  }
  ~PhaseAligner() { delete ctx_; }
  void alignRegistered(const CloudView& prev, const CloudView& reg) {
    phgpu_cloud a = prev.c(), b = reg.c();
    detail::check(phgpu_voxelize(ctx_->get(), &a, 0, nullptr), ctx_->get(), "phgpu_voxelize");
    detail::check(phgpu_voxelize(ctx_->get(), &b, 1, nullptr), ctx_->get(), "phgpu_voxelize");
    detail::check(phgpu_spatial_correlate_voxelized(ctx_->get()), ctx_->get(), "phgpu_spatial_correlate");
  }
  std::vector<double> getCorrelation() const {
    std::vector<double> out(phgpu_spatial_correlation_size(ctx_->get()));
    detail::check(phgpu_spatial_result(ctx_->get(), nullptr, nullptr, out.data()), ctx_->get(),
                  "phgpu_spatial_result");
    return out;
  }
  // n_voxels + 2 zero padding (phase-aligner.cc:137-139)
  uint32_t getNumberOfVoxels() const noexcept { return prm_.spatial_n_voxels + 2 * prm_.spatial_zero_padding; }
  // the reference returns the int bounds through uint32 (phase-aligner.cc:141-147)
  uint32_t getLowerBound() const noexcept { return (uint32_t)prm_.spatial_discretize_lower; }
  uint32_t getUpperBound() const noexcept { return (uint32_t)prm_.spatial_discretize_upper; }

 private:
  phgpu_params prm_;
  detail::Context* ctx_ = nullptr;
};

// SphOptRegistration::registerPointCloud(prev = target, cur = source).
class SphOptRegistration {
 public:
  explicit SphOptRegistration(const phgpu_params& base = default_params()) : ctx_(base) {}
  phgpu_pose registerPointCloud(const CloudView& cloud_prev, const CloudView& cloud_cur) {
    phgpu_cloud t = cloud_prev.c(), s = cloud_cur.c();
    phgpu_pose pose;
    detail::check(phgpu_register_pair(ctx_.get(), &t, &s, &pose), ctx_.get(), "phgpu_register_pair");
    return pose;
  }

 private:
  detail::Context ctx_;
};

// SphRegistration::registerPointCloud (sph-registration.cc:82-198): rotation
// from the single 0.6 intensity + 0.4 range signal of the sampled directions
// with the plain SphericalCorrelation, then the PhaseAligner translation of
// the rotated cloud (prev = target, cur = source).
class SphRegistration {
 public:
  explicit SphRegistration(const phgpu_params& base = default_params()) : ctx_(mix_params(base)) {}
  phgpu_pose registerPointCloud(const CloudView& cloud_prev, const CloudView& cloud_cur) {
    phgpu_cloud t = cloud_prev.c(), s = cloud_cur.c();
    phgpu_pose pose;
    detail::check(phgpu_register_pair(ctx_.get(), &t, &s, &pose), ctx_.get(), "phgpu_register_pair");
    return pose;
  }

 private:
  static phgpu_params mix_params(phgpu_params p) {
    p.spherical_fusion = PHGPU_FUSION_MIX;
    return p;
  }
  detail::Context ctx_;
};

// ------------------------------------------------------------------ S^2 sampling

// SphericalSampler::sampleUniformly (spherical-sampler.cc:20-27): the 2B x 2B
// Driscoll-Healy directions, [theta][phi] order, each sampled by its nearest
// point of the cloud's projection on the unit sphere.  The rejection radius
// comes from the parameters as in a context.
// ZScorePeakExtraction (phaser_core/include/phaser/backend/uncertainty/
// z-score-peak-extraction.h): smoothed z-score peaks of a correlation vector,
// the parameters defaulting to the reference's z_score_* flags.
class ZScorePeakExtraction {
 public:
  ZScorePeakExtraction() { phgpu_zscore_params_default(&p_); }
  void extractPeaks(const std::vector<double>& corr, std::set<uint32_t>* peaks) {
    std::vector<uint32_t> out(corr.empty() ? 1 : corr.size());
    uint64_t n = 0;
    const int rc = phgpu_zscore_peaks(corr.data(), corr.size(), &p_, out.data(), out.size(), &n);
    if (rc != PHGPU_OK) throw std::runtime_error("phgpu_zscore_peaks failed");
    peaks->clear();
    peaks->insert(out.begin(), out.begin() + n);
  }
  double getLagPercentile() const { return p_.lag_percentile; }
  double& getLagPercentile() { return p_.lag_percentile; }
  double getScoreThreshold() const { return p_.threshold; }
  double& getScoreThreshold() { return p_.threshold; }
  double getInfluence() const { return p_.influence; }
  double& getInfluence() { return p_.influence; }
  uint32_t getMaxLag() const { return p_.lag_max; }
  uint32_t& getMaxLag() { return p_.lag_max; }

 private:
  phgpu_zscore_params p_;
};

class SphericalSampler {
 public:
  explicit SphericalSampler(int bandwith, const phgpu_params& base = default_params()) : base_(base) {
    initialize(bandwith);
  }
  void initialize(int bandwith) {
    phgpu_params p = base_;
    p.spherical_bandwidth = (uint32_t)bandwith;
    p.spherical_zero_padding = 0;
    ctx_.reset(new detail::Context(p));
    bw_ = bandwith;
  }
  int getInitializedBandwith() const noexcept { return bw_; }
  void sampleUniformly(const CloudView& cloud, std::vector<FunctionValue>* grid) {
    phgpu_cloud c = cloud.c();
    detail::check(phgpu_sample_s2(ctx_->get(), &c, 0), ctx_->get(), "phgpu_sample_s2");
    const size_t nq = (size_t)4 * bw_ * bw_;
    std::vector<double> v(4 * nq);
    std::vector<int32_t> nn(nq);
    detail::check(phgpu_get_samples(ctx_->get(), 0, v.data(), nn.data()), ctx_->get(), "phgpu_get_samples");
    grid->assign(nq, FunctionValue());
    for (size_t q = 0; q < nq; ++q) {
      FunctionValue& f = (*grid)[q];
      f.range = v[q];
      f.intensity = v[nq + q];
      f.reflectivity = v[2 * nq + q];
      f.ambient = v[3 * nq + q];
      f.nn_index = nn[q];
    }
  }

 private:
  phgpu_params base_;
  std::unique_ptr<detail::Context> ctx_;
  int bw_ = 0;
};

// ------------------------------------------------------------------ ingest

// The fields PlyHelper reads (ply-helper.cc:26-64), narrowed to float as the
// reference's cloud does: x, y, z, intensity interleaved, and the optional
// reflectivity, ambient ("noise") and range (empty when the file lacks them).
struct PlyPointCloud {
  std::vector<float> xyzi;  // [n][4]
  std::vector<float> reflectivity, ambient, range;
  size_t size() const noexcept { return xyzi.size() / 4; }
  const std::vector<float>& getReflectivities() const noexcept { return reflectivity; }
  const std::vector<float>& getAmbientPoints() const noexcept { return ambient; }
  const std::vector<float>& getRange() const noexcept { return range; }
  // x, y, z, intensity + optional channels as the aligner / registration take them
  CloudView view() const {
    CloudView v;
    v.xyzi = xyzi.data();
    v.reflectivity = reflectivity.empty() ? nullptr : reflectivity.data();
    v.ambient = ambient.empty() ? nullptr : ambient.data();
    v.n_points = (uint32_t)size();
    return v;
  }
};

// PlyHelper::readPlyFromFile; the field names default to the reference's
// --phaser_ply_{intensity,reflectivity,ambient,range}_str flags.
class PlyHelper {
 public:
  explicit PlyHelper(std::string intensity = "intensity", std::string reflectivity = "reflectivity",
                     std::string ambient = "noise", std::string range = "range")
      : names_{std::move(intensity), std::move(reflectivity), std::move(ambient), std::move(range)} {}
  PlyPointCloud readPlyFromFile(const std::string& filename) const {
    const char* names[4] = {names_[0].c_str(), names_[1].c_str(), names_[2].c_str(), names_[3].c_str()};
    uint32_t n = 0, present = 0;
    ply_check(phgpu_ply_info(filename.c_str(), names, &n, &present));
    PlyPointCloud pc;
    pc.xyzi.resize((size_t)n * 4);
    if (present & PHGPU_PLY_REFLECTIVITY) pc.reflectivity.resize(n);
    if (present & PHGPU_PLY_AMBIENT) pc.ambient.resize(n);
    if (present & PHGPU_PLY_RANGE) pc.range.resize(n);
    uint32_t got = 0;
    ply_check(phgpu_ply_read(filename.c_str(), names, pc.xyzi.data(),
                             pc.reflectivity.empty() ? nullptr : pc.reflectivity.data(),
                             pc.ambient.empty() ? nullptr : pc.ambient.data(),
                             pc.range.empty() ? nullptr : pc.range.data(), n, &got));
    return pc;
  }

 private:
  static void ply_check(int rc) {
    if (rc != PHGPU_OK) throw std::runtime_error(std::string("phgpu_ply: ") + phgpu_ply_last_error());
  }
  std::string names_[4];
};

// VoxelGridCmd::execute (voxel-grid-cmd.cc:11-22): pcl::VoxelGrid with leaf
// --phaser_voxel_grid_leaf_size (0.25) on the GPU, filtering the cloud in
// place (reflectivity and ambient, when present, are averaged over the same
// leaves; range is per raw point and is dropped).
class VoxelGridCmd {
 public:
  explicit VoxelGridCmd(float leaf_size = 0.25f, int32_t device = 0) : leaf_(leaf_size), device_(device) {}
  ~VoxelGridCmd() {
    if (vg_) phgpu_voxel_grid_destroy(vg_);
  }
  VoxelGridCmd(const VoxelGridCmd&) = delete;
  VoxelGridCmd& operator=(const VoxelGridCmd&) = delete;
  void execute(PlyPointCloud& cloud) {
    const uint32_t n = (uint32_t)cloud.size();
    if (!vg_ || n > cap_) {
      if (vg_) phgpu_voxel_grid_destroy(vg_);
      vg_ = nullptr;
      cap_ = std::max<uint32_t>(n, 1u);
      if (phgpu_voxel_grid_create(cap_, device_, &vg_) != PHGPU_OK)
        throw std::runtime_error("phgpu_voxel_grid_create failed");
    }
    phgpu_cloud in = cloud.view().c();
    std::vector<float> xyzi((size_t)n * 4), refl(cloud.reflectivity.empty() ? 0 : n),
        amb(cloud.ambient.empty() ? 0 : n);
    const float leaf[3] = {leaf_, leaf_, leaf_};
    uint32_t m = 0;
    if (phgpu_voxel_grid_filter(vg_, &in, leaf, 0, xyzi.data(), refl.empty() ? nullptr : refl.data(),
                                amb.empty() ? nullptr : amb.data(), 0, &m) != PHGPU_OK)
      throw std::runtime_error(std::string("phgpu_voxel_grid_filter: ") + phgpu_voxel_grid_last_error(vg_));
    xyzi.resize((size_t)m * 4);
    cloud.xyzi = std::move(xyzi);
    if (!refl.empty()) refl.resize(m);
    if (!amb.empty()) amb.resize(m);
    cloud.reflectivity = std::move(refl);
    cloud.ambient = std::move(amb);
    cloud.range.clear();
  }

 private:
  float leaf_;
  int32_t device_;
  phgpu_voxel_grid* vg_ = nullptr;
  uint32_t cap_ = 0;
};

}  // namespace phaser_gpu

#endif  // PHASER_GPU_HPP_
