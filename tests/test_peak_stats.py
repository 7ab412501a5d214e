"""Peak-neighbourhood statistics (bingham_/gaussian_peak_neighbors > 0):
the host functions of the C ABI against the oracle's restatement and against a
numpy restatement of the reference's formulas (no GPU needed).

Tolerance: both sides are FP64; eigenvectors are compared up to sign."""
import itertools

import numpy as np
import pytest

from oracle import oracle as O


@pytest.fixture(scope="module")
def nat():
    from phaser_b200 import native
    native.load()
    return native


def test_window_rule(nat):
    # calculateStartEndNeighbor: one-sided at both ends of the volume
    for index, n, k in itertools.product([0, 1, 2, 5, 97, 98, 99], [100], [0, 1, 3, 7]):
        assert nat.peak_window(index, n, k) == O.peak_window(index, n, k)
    assert nat.peak_window(5, 100, 3) == (2, 7)
    assert nat.peak_window(1, 100, 3) == (1, 4)
    assert nat.peak_window(98, 100, 3) == (95, 4)


def _numpy_bingham(values, first, bw):
    q = np.array([O.bin_to_pose(first + i, bw)[1] for i in range(len(values))])
    w = np.asarray(values, float)
    if len(w) > 1:
        w = w / w.sum()
    C = (q * w[:, None]).T @ q
    ev, V = np.linalg.eigh(0.5 * (C + C.T))
    return V[:, -1], ev / ev.sum()


@pytest.mark.parametrize("bw,k", [(8, 1), (8, 3), (100, 2), (100, 5)])
def test_bingham_peak_matches_oracle_and_numpy(nat, bw, k):
    rng = np.random.default_rng(bw + k)
    n = (2 * bw) ** 3
    index = int(rng.integers(k, n - k))
    first, count = nat.peak_window(index, n, k)
    values = rng.random(count) + 0.05
    mode, omega, xyz = nat.bingham_peak(values, first, bw)
    omode, oomega, oxyz = O.bingham_peak(values, first, bw)
    np.testing.assert_allclose(mode, omode, atol=1e-12)
    np.testing.assert_allclose(omega, oomega, atol=1e-12)
    np.testing.assert_allclose(xyz, oxyz, atol=1e-12)
    nmode, nomega = _numpy_bingham(values, first, bw)
    assert abs(abs(float(np.dot(mode, nmode))) - 1.0) < 1e-12
    np.testing.assert_allclose(omega, nomega, atol=1e-12)
    assert mode[0] >= 0


def test_bingham_single_bin_is_the_bin(nat):
    # neighbours = 0: the fit of one sample returns that bin's rotation
    bw, b = 100, 4903744
    mode, omega, xyz = nat.bingham_peak([0.7], b, bw)
    _, q, e = O.bin_to_pose(b, bw)
    assert abs(abs(float(np.dot(mode, q))) - 1.0) < 1e-12
    np.testing.assert_allclose(omega, [0, 0, 0, 1], atol=1e-12)
    np.testing.assert_allclose(xyz, e, atol=1e-9)


def _numpy_gaussian(values, first, N, lo, hi):
    t = np.array([[O.translation_from_index(s, N, lo, hi) for s in O.ind2sub(first + i, N, N)]
                  for i in range(len(values))])
    w = np.asarray(values, float) / np.sum(values)
    mu = t.T @ w
    z = (t - mu) * np.sqrt(w)[:, None]
    return mu, z.T @ z


@pytest.mark.parametrize("N,k", [(64, 1), (64, 4), (200, 3), (200, 10)])
def test_gaussian_peak_matches_oracle_and_numpy(nat, N, k):
    rng = np.random.default_rng(N * 3 + k)
    n = N ** 3
    index = int(rng.integers(0, n))
    first, count = nat.peak_window(index, n, k)
    values = rng.random(count) + 0.05
    mean, cov = nat.gaussian_peak(values, first, N, -10, 10)
    omean, ocov = O.gaussian_peak(values, first, N, -10, 10)
    np.testing.assert_allclose(mean, omean, atol=1e-12)
    np.testing.assert_allclose(cov, ocov, atol=1e-12)
    nmean, ncov = _numpy_gaussian(values, first, N, -10, 10)
    np.testing.assert_allclose(mean, nmean, atol=1e-12)
    np.testing.assert_allclose(cov, ncov, atol=1e-12)


def test_gaussian_negative_weight_gives_nan_like_the_reference(nat):
    # Gaussian::setMeanAndCov scales by sqrt(w): a negative weight yields NaN
    mean, cov = nat.gaussian_peak([1.0, -0.2, 0.5], 1000, 64, -10, 10)
    omean, ocov = O.gaussian_peak([1.0, -0.2, 0.5], 1000, 64, -10, 10)
    np.testing.assert_allclose(mean, omean, atol=1e-12)
    assert np.isnan(cov).any() and np.isnan(ocov).any()


def test_invalid_weights_rejected(nat):
    with pytest.raises(nat.PhgpuError):
        nat.gaussian_peak([0.0, 0.0], 0, 8, -1, 1)
    with pytest.raises(nat.PhgpuError):
        nat.bingham_peak([0.0, 0.0], 0, 8)


@pytest.mark.gpu
@pytest.mark.parametrize("rot_k,trans_k", [(2, 3), (5, 0), (0, 6)])
def test_register_pair_with_peak_neighbours(nat, rot_k, trans_k):
    """With neighbours the pose is the Bingham mode and the Gaussian mean.
    Tolerances: the GPU weights are the FP32 volumes (the oracle's FP64), so
    angles agree to 1e-5 rad, translations to 1e-4 m, statistics to 1e-4
    relative; bins and voxels are identical."""
    from phaser_b200 import scene
    w = scene.WORKLOADS[0]
    pair = scene.workload_pair(0, 0)
    c = nat.Context(spherical_bandwidth=w["bw"], spatial_n_voxels=w["n_voxels"], spatial_discretize_lower=w["lo"],
                    spatial_discretize_upper=w["hi"], rot_peak_neighbors=rot_k, trans_peak_neighbors=trans_k)
    pose = c.register_pair((pair.target.xyzi, None), (pair.source.xyzi, None))
    c.close()
    opose, omega, cov = O.register_pair(pair.target.xyzi, None, pair.source.xyzi, None, w["bw"], w["n_voxels"],
                                        w["lo"], w["hi"], rot_k=rot_k, trans_k=trans_k, want_stats=True)
    assert pose.rot_bin == opose.rot_bin
    assert pose.voxel == opose.voxel
    np.testing.assert_allclose(list(pose.xyz), list(opose.xyz), atol=1e-5)
    assert abs(abs(float(np.dot(list(pose.quat), list(opose.quat)))) - 1.0) < 1e-8
    np.testing.assert_allclose(list(pose.trans), list(opose.trans), atol=1e-4)
    np.testing.assert_allclose(list(pose.rot_omega), omega, atol=1e-4)
    np.testing.assert_allclose(np.array(pose.trans_cov).reshape(3, 3), cov, atol=1e-4 * max(1e-3, np.abs(cov).max()))
