"""The oracle's literal restatement of the zero-padded spatial correlation
(orc_spatial_correlation_padded; spatial-correlation.cc:11-45,142-161,
163-230, spatial-correlation-laplace.cc:17-50, spatial-correlation-low-pass.cc
:40-69) checked on CPU: with padding 0 it reduces to the unpadded
restatements bit for bit; the reported correlation length follows the
reference's double-precision truncation; the Laplace mode carries the
previous call's last channel through the shifted buffer's tail, the plain
mode carries nothing."""
import numpy as np
import pytest

from oracle import oracle as O


@pytest.mark.parametrize("N", [6, 7, 8])
def test_padding_zero_reduces_to_unpadded(N):
    rng = np.random.default_rng(N)
    f = rng.standard_normal((4, N ** 3))
    g = rng.standard_normal((4, N ** 3))
    v, size = O.spatial_correlation_padded(f, g, N, 0, mode=1)
    assert size == N ** 3
    assert np.array_equal(v, O.spatial_correlation(f, g, N, laplace=True))
    v, _ = O.spatial_correlation_padded(f, g, N, 0, mode=0)
    assert np.array_equal(v, O.spatial_correlation(f[:1], g[:1], N, laplace=False))
    v, _ = O.spatial_correlation_padded(f, g, N, 0, mode=2, lower=1, upper=N - 2)
    assert np.array_equal(v, O.spatial_correlation_lowpass(f[1], g[1], N, 1, N - 2))


def test_correlation_length_truncation():
    # uint32(N^3 * ((N + 2p) / N)^3) in double: (N + 2p)^3 - 1 for many pairs
    rng = np.random.default_rng(1)
    f = rng.standard_normal((1, 27))
    seen = set()
    for N, p in [(3, 4), (5, 1), (3, 1), (4, 2), (6, 8)]:
        fN = rng.standard_normal((1, N ** 3))
        _, size = O.spatial_correlation_padded(fN, fN, N, p, mode=0)
        r = (N + 2 * p) / float(N)
        assert size == int(float(N ** 3) * (r * r * r))
        seen.add((N + 2 * p) ** 3 - size)
    assert seen == {0, 1}


def test_laplace_state_carries_last_channel():
    N, p = 6, 2
    rng = np.random.default_rng(7)
    f1, g1 = rng.standard_normal((4, N ** 3)), rng.standard_normal((4, N ** 3))
    f2, g2 = rng.standard_normal((4, N ** 3)), rng.standard_normal((4, N ** 3))
    st = O.new_padded_state(N)
    O.spatial_correlation_padded(f1, g1, N, p, mode=1, state=st)
    after, _ = O.spatial_correlation_padded(f2, g2, N, p, mode=1, state=st)
    fresh, _ = O.spatial_correlation_padded(f2, g2, N, p, mode=1)
    assert not np.allclose(after, fresh)  # the first channel read the previous call's tail
    # a zero last channel leaves a zero tail for the next call
    f1[3] = 0
    g1[3] = 0
    st = O.new_padded_state(N)
    O.spatial_correlation_padded(f1, g1, N, p, mode=1, state=st)
    after, _ = O.spatial_correlation_padded(f2, g2, N, p, mode=1, state=st)
    assert np.array_equal(after, fresh)
    # the plain correlation never shifts: no state
    st = O.new_padded_state(N)
    O.spatial_correlation_padded(f1, g1, N, p, mode=0, state=st)
    a, _ = O.spatial_correlation_padded(f2, g2, N, p, mode=0, state=st)
    b, _ = O.spatial_correlation_padded(f2, g2, N, p, mode=0)
    assert np.array_equal(a, b)
