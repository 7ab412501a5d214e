// Smoothed z-score peak extraction (phgpu_zscore_peaks): the reference's
// ZScorePeakExtraction (phaser_core/src/backend/uncertainty/
// z-score-peak-extraction.cc:42-112), a consumer of a correlation volume.
//
// The scan is sequential by construction -- a damped peak changes the values
// the following windows average -- so it runs on the host in FP64 over a
// volume the caller has read back (phgpu_sph_result / phgpu_spatial_result
// with the volume kept), like the Bingham and Gaussian fits of the peak
// neighbourhoods.  The window sums run in index order; the reference takes
// them with Eigen array reductions, whose (vectorised) summation order is not
// pinned here, so a value within rounding of the threshold may classify
// differently.
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/phaser_gpu.h"

int phgpu_zscore_params_default(phgpu_zscore_params* p) {
  if (!p) return PHGPU_ERR_INVALID;
  // z-score-peak-extraction.cc:11-25
  p->lag_percentile = 0.05;
  p->lag_max = 20;
  p->threshold = 4.33;
  p->influence = 0.05;
  p->filter_threshold = 0.405;
  return PHGPU_OK;
}

namespace {

// Mean and sample standard deviation (divisor lag - 1) of x[start, start + lag).
void window_stats(const double* x, size_t start, size_t lag, double* avg, double* dev) {
  double s = 0.0;
  for (size_t k = 0; k < lag; ++k) s += x[start + k];
  const double m = s / (double)lag;
  double q = 0.0;
  for (size_t k = 0; k < lag; ++k) {
    const double d = x[start + k] - m;
    q += d * d;
  }
  *avg = m;
  *dev = std::sqrt(q / ((double)lag - 1.0));
}

}  // namespace

int phgpu_zscore_peaks(const double* values, uint64_t n, const phgpu_zscore_params* prm, uint32_t* peaks,
                       uint64_t capacity, uint64_t* n_peaks) {
  if (!prm || !n_peaks || (n && !values) || (capacity && !peaks)) return PHGPU_ERR_INVALID;
  if (!(prm->lag_percentile > 0.0 && prm->lag_percentile < 1.0) || !(prm->threshold > 0.0) ||
      !(prm->influence >= 0.0 && prm->influence <= 1.0) || n > 0xffffffffull)
    return PHGPU_ERR_INVALID;
  *n_peaks = 0;
  // extractPeaks: lag = min(lag_max, (uint32)(n * lag_percentile))
  const uint32_t by_share = (uint32_t)((double)n * prm->lag_percentile);
  const size_t lag = by_share < prm->lag_max ? by_share : prm->lag_max;
  // calculateSmoothedZScore: nothing when n <= lag + 2
  if (n <= (uint64_t)lag + 2) return PHGPU_OK;
  std::vector<double> x(values, values + n);
  double avg, dev;
  window_stats(x.data(), 0, lag, &avg, &dev);
  const double keep = 1.0 - prm->influence;
  uint64_t count = 0;
  for (size_t i = lag + 1; i < n; ++i) {
    const double v = x[i];
    if (v <= prm->filter_threshold) continue;  // skips the window update too
    if (std::fabs(v - avg) > prm->threshold * dev) {
      if (v >= avg) {
        if (count < capacity) peaks[count] = (uint32_t)i;
        ++count;
      }
      x[i] = prm->influence * v + keep * x[i - 1];
    }
    window_stats(x.data(), i - lag, lag, &avg, &dev);
  }
  *n_peaks = count;
  return count > capacity ? PHGPU_ERR_LIMIT : PHGPU_OK;
}
