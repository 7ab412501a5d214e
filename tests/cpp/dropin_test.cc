// Drives the C++ drop-ins of include/phaser_gpu.hpp the way phaser_core's
// registration calls the reference classes; prints one line per check.
// Built and run by tests/test_cpp_dropin.py.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "phaser_gpu.hpp"

int main() {
  using namespace phaser_gpu;
  // spatial delta known answer (phaser_core/test/translation-alignment/
  // spatial-correlation-test.cc:59-79): f[0] = 1, g[1] = 1 -> Ind2Sub (0, 2, 0)
  {
    std::vector<double> f(27, 0.0), g(27, 0.0);
    f[0] = 1.0;
    g[1] = 1.0;
    SpatialCorrelation corr(3u);
    double* c = corr.correlateSignals({f.data()}, {g.data()});
    size_t best = 0;
    for (size_t i = 1; i < 27; ++i)
      if (c[i] > c[best]) best = i;
    const unsigned x = (best / 3) % 3, y = best % 3, z = best / 9;
    std::printf("spatial_delta %u %u %u\n", x, y, z);
    if (!(x == 0 && y == 2 && z == 0)) return 1;
  }
  // Laplace spherical correlation of 4 channels through the drop-in
  {
    const uint32_t bw = 8;
    std::vector<SampledSignal> f(4, SampledSignal(4 * bw * bw)), g(4, SampledSignal(4 * bw * bw));
    unsigned s = 12345;
    for (auto* side : {&f, &g})
      for (auto& ch : *side)
        for (auto& v : ch) {
          s = s * 1103515245u + 12345u;
          v = ((s >> 8) & 0xffff) / 65535.0 - 0.5;
        }
    SphericalCorrelationLaplace corr(bw);
    corr.correlateSampledSignals(f, g);
    const std::vector<double> vol = corr.getCorrelation();
    size_t best = 0;
    for (size_t i = 1; i < vol.size(); ++i)
      if (vol[i] > vol[best]) best = i;
    std::printf("sph_laplace_bin %zu %u bw_out %u\n", best, corr.getPeakBin(), corr.getBandwidth());
    if (best != corr.getPeakBin() || vol.size() != 8u * bw * bw * bw) return 2;
  }
  // zero padding: the correlation covers (n + 2 pad)^3 voxels, of which the
  // reference reports uint32(n^3 ((n + 2 pad) / n)^3)
  {
    std::vector<double> f(27, 0.0), g(27, 0.0);
    f[0] = 1.0;
    g[1] = 1.0;
    SpatialCorrelation corr(3u, 1u);
    const double ratio = 5.0 / 3.0;
    const uint32_t want = (uint32_t)(27.0 * (ratio * ratio * ratio));
    corr.correlateSignals({f.data()}, {g.data()});
    std::printf("padded_size %u %u\n", corr.getCorrelationSize(), want);
    if (corr.getCorrelationSize() != want || corr.getZeroPadding() != 1u) return 3;
  }
  // invalid configuration is reported as an exception, not an abort
  try {
    SpatialCorrelation bad(1000u, 20u);  // n + 2 pad > 1024
    return 4;
  } catch (const std::runtime_error&) {
    std::printf("invalid_configuration_rejected\n");
  }
  // SphericalSampler on a one-point cloud: every direction's nearest point is
  // that point (the default rejection radius is 1000 m), range |p| = 3
  {
    const float xyzi[4] = {3.0f, 0.0f, 0.0f, 5.0f};
    CloudView cv;
    cv.xyzi = xyzi;
    cv.n_points = 1;
    SphericalSampler sampler(8);
    std::vector<FunctionValue> grid;
    sampler.sampleUniformly(cv, &grid);
    std::printf("sampler %zu bw %d\n", grid.size(), sampler.getInitializedBandwith());
    if (grid.size() != 4u * 8u * 8u) return 7;
    for (const FunctionValue& f : grid)
      if (f.nn_index != 0 || f.getAveragedRange() != 3.0 || f.getAveragedIntensity() != 5.0 ||
          f.getAveragedReflectivity() != 0.0)
        return 8;
  }
  // SphRegistration's single signal: SphericalCorrelation::correlateSignals on
  // the sampled FunctionValues of two clouds gives the bin SphRegistration
  // registers them with; the Laplace class refuses the single signal
  {
    std::vector<float> a, b;
    unsigned s = 777;
    for (int i = 0; i < 3000; ++i) {
      float p[4];
      for (float& v : p) {
        s = s * 1103515245u + 12345u;
        v = ((s >> 8) & 0xffff) / 65535.0f * 8.0f - 4.0f;
      }
      p[3] = std::fabs(p[3]) / 4.0f;
      a.insert(a.end(), p, p + 4);
      b.insert(b.end(), {p[1], -p[0], p[2] + 0.5f, p[3]});  // rotated by 90 degrees about z, shifted
    }
    CloudView ca, cb;
    ca.xyzi = a.data();
    ca.n_points = 3000;
    cb.xyzi = b.data();
    cb.n_points = 3000;
    phgpu_params prm = default_params();
    prm.spherical_bandwidth = 16;
    prm.spatial_n_voxels = 32;
    prm.spatial_discretize_lower = -10;
    prm.spatial_discretize_upper = 10;
    SphericalSampler sampler(16, prm);
    std::vector<FunctionValue> fa, fb;
    sampler.sampleUniformly(ca, &fa);
    sampler.sampleUniformly(cb, &fb);
    SphericalCorrelation corr(16u, 0u, prm);
    corr.correlateSignals(fa, fb);
    SphRegistration reg(prm);
    const phgpu_pose pose = reg.registerPointCloud(ca, cb);
    std::printf("sph_registration_bin %u %u\n", corr.getPeakBin(), pose.rot_bin);
    if (corr.getPeakBin() != pose.rot_bin) return 9;
    SphericalCorrelationLaplace lap(16u, 0u, prm);
    try {
      lap.correlateSignals(fa, fb);
      return 10;
    } catch (const std::invalid_argument&) {
      std::printf("laplace_refuses_single_signal\n");
    }
  }
  // VoxelGridCmd on a cloud of three points: leaves (0,0,0) and (2,0,0) at
  // leaf 0.25 (grid anchored at floor(min / leaf)); each leaf's mean is the
  // in-order float sum divided by the count
  {
    PlyPointCloud pc;
    pc.xyzi = {0.1f, 0.1f, 0.1f, 1.0f, 0.2f, 0.1f, 0.1f, 3.0f, 0.6f, 0.1f, 0.1f, 5.0f};
    VoxelGridCmd cmd(0.25f);
    cmd.execute(pc);
    float sx = 0.0f, sy = 0.0f;
    sx += 0.1f;
    sx += 0.2f;
    sy += 0.1f;
    sy += 0.1f;
    const float want[8] = {sx / 2.0f, sy / 2.0f, sy / 2.0f, 2.0f, 0.6f, 0.1f, 0.1f, 5.0f};
    std::printf("voxel_grid %zu\n", pc.size());
    if (pc.size() != 2u) return 5;
    for (int k = 0; k < 8; ++k)
      if (pc.xyzi[k] != want[k]) return 6;
  }
  {
    // ZScorePeakExtraction: spikes on a flat signal (the reference's flags)
    std::vector<double> corr(2000);
    for (size_t i = 0; i < corr.size(); ++i) corr[i] = 1.0 + 1e-3 * std::sin((double)i);
    corr[300] = corr[777] = corr[1500] = 50.0;
    phaser_gpu::ZScorePeakExtraction z;
    std::set<uint32_t> peaks;
    z.extractPeaks(corr, &peaks);
    std::printf("zscore_peaks %zu\n", peaks.size());
    if (peaks != std::set<uint32_t>{300u, 777u, 1500u}) return 7;
    z.getScoreThreshold() = 1e9;  // nothing stands out any more
    z.extractPeaks(corr, &peaks);
    if (!peaks.empty()) return 8;
  }
  std::printf("ok\n");
  return 0;
}
