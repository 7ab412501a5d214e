"""Smoothed z-score peak extraction (phgpu_zscore_peaks, the reference's
ZScorePeakExtraction, z-score-peak-extraction.cc:42-112) against the oracle's
restatement: identical signal indices on seeded vectors, known answers on a
flat signal with spikes, the reference's parameter checks and the short-input
rule.  Host code: runs without a GPU."""
import numpy as np
import pytest

from oracle import oracle as O


@pytest.fixture(scope="module")
def nat():
    from phaser_b200 import native
    native.load()
    return native


@pytest.mark.parametrize("seed,n", [(0, 50), (1, 1000), (2, 40000), (3, 8 * 32 ** 3)])
def test_matches_oracle(nat, seed, n):
    rng = np.random.default_rng(seed)
    v = rng.gamma(2.0, 1.0, n)
    v[rng.choice(n, max(n // 500, 3), replace=False)] += rng.uniform(5, 50, max(n // 500, 3))
    got = nat.zscore_peaks(v)
    want = O.zscore_peaks(v)
    assert got.dtype == np.uint32
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("kw", [dict(threshold=2.0), dict(influence=0.5), dict(lag_max=5),
                                dict(lag_percentile=0.001, lag_max=1000), dict(filter_threshold=-1e9)])
def test_parameters_match_oracle(nat, kw):
    rng = np.random.default_rng(7)
    v = rng.standard_normal(20000) + 3.0
    v[::997] += 20.0
    np.testing.assert_array_equal(nat.zscore_peaks(v, **kw), O.zscore_peaks(v, **kw))


def test_spikes_on_a_flat_signal(nat):
    v = np.ones(2000)
    v += 1e-3 * np.sin(np.arange(2000))  # a non-zero window deviation
    spikes = [300, 777, 1500]
    v[spikes] = 50.0
    assert list(nat.zscore_peaks(v)) == spikes
    # values at or below the filter threshold are never signals
    assert list(nat.zscore_peaks(v, filter_threshold=60.0)) == []


def test_short_input_and_checks(nat):
    from phaser_b200.native import PhgpuError
    # lag = min(20, (uint32)(n * 0.05)); n <= lag + 2 gives no peaks
    assert nat.zscore_peaks(np.array([1.0, 100.0])).size == 0
    assert nat.zscore_peaks(np.zeros(0)).size == 0
    for kw in (dict(lag_percentile=0.0), dict(lag_percentile=1.0), dict(threshold=0.0), dict(influence=1.5)):
        with pytest.raises(PhgpuError):
            nat.zscore_peaks(np.ones(100), **kw)
