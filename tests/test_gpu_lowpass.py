"""Low-pass correlation variants against the oracle's literal restatement of
SphericalCorrelationLowPass / SpatialCorrelationLowPass (FFT shifts of the
coefficient arrays, band / cube index sets, shifts back).

Tolerance: FP32 volumes within relative L2 1e-5 of the FP64 oracle; the argmax
is compared where the top value is separated from the second by more than
that tolerance."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

REL_L2 = 1e-5


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


def distinct_max(v):
    s = np.sort(np.asarray(v))
    return s[-1] - s[-2] > 1e-4 * max(abs(s[-1]), 1e-30)


@pytest.mark.parametrize("bw,pad,lo,hi", [(8, 0, 0, 100000), (8, 0, 5, 40), (16, 0, 64, 192), (16, 3, 10, 200),
                                          (12, 0, 0, 30)])
def test_spherical_lowpass_vs_oracle(bw, pad, lo, hi):
    from phaser_b200.core import SphericalCorrelationLowPass
    rng = np.random.default_rng(bw * 1000 + lo + hi)
    f = rng.standard_normal((3, 4 * bw * bw))
    g = rng.standard_normal((3, 4 * bw * bw))
    corr = SphericalCorrelationLowPass(bw, pad, lower=lo, upper=hi)
    corr.correlateSampledSignals(list(f), list(g))
    vol = corr.getCorrelation()
    ref = O.spherical_correlation_lowpass(f[0], g[0], bw, lo, hi, bw_out=bw + pad)
    assert rel_l2(vol, ref) <= REL_L2
    if distinct_max(ref):
        assert int(np.argmax(vol)) == O.argmax(ref)


@pytest.mark.parametrize("N,lo,hi", [(6, 0, 100000), (16, 1, 14), (16, 2, 8), (9, 0, 5), (30, 3, 25), (64, 8, 40)])
def test_spatial_lowpass_vs_oracle(N, lo, hi):
    from phaser_b200.core import SpatialCorrelationLowPass
    rng = np.random.default_rng(N * 100 + lo + hi)
    f = rng.standard_normal((2, N ** 3))
    g = rng.standard_normal((2, N ** 3))
    corr = SpatialCorrelationLowPass(N, 0, lower=lo, upper=hi)
    assert corr.getUpperBound() == min(hi, N)
    vol = corr.correlateSignals(list(f), list(g))
    ref = O.spatial_correlation_lowpass(f[1], g[1], N, lo, min(hi, N))
    assert rel_l2(vol, ref) <= REL_L2
    if distinct_max(ref):
        assert int(np.argmax(vol)) == O.argmax(ref)


def test_spatial_lowpass_needs_channel_one():
    from phaser_b200 import native as nat
    from phaser_b200.core import SpatialCorrelationLowPass
    corr = SpatialCorrelationLowPass(8, 0, lower=1, upper=6)
    with pytest.raises(nat.PhgpuError):
        corr.correlateSignals([np.ones(512)], [np.ones(512)])
