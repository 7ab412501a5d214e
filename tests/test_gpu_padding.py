"""Zero-padded spatial correlation on the GPU against the oracle's literal
restatement (orc_spatial_correlation_padded): plain, Laplace and low-pass
modes, odd and even N, the reference's correlation length, the Laplace
state carried from one call to the next, and a padded registration whose
voxel and translation decode on N + 2 pad voxels.

Tolerance: FP32 volumes within relative L2 1e-5 of the FP64 oracle; argmax
compared where the top value is separated from the second by more than 1e-4
relative."""
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


def check(vol, ref, size):
    assert len(vol) == size
    assert rel_l2(vol, ref[:size]) <= REL_L2
    if distinct_max(ref[:size]):
        assert int(np.argmax(vol)) == int(np.argmax(ref[:size]))


@pytest.mark.parametrize("N,pad", [(6, 1), (8, 2), (9, 2), (16, 3), (30, 5), (64, 4)])
def test_laplace_padded_vs_oracle(N, pad):
    from phaser_b200.core import SpatialCorrelationLaplace
    rng = np.random.default_rng(N * 10 + pad)
    f = rng.standard_normal((4, N ** 3))
    g = rng.standard_normal((4, N ** 3))
    corr = SpatialCorrelationLaplace(N, pad)
    vol = corr.correlateSignals(list(f), list(g))
    ref, size = O.spatial_correlation_padded(f, g, N, pad, mode=1)
    assert corr.getCorrelationSize() == size
    check(vol, ref, size)


@pytest.mark.parametrize("N,pad", [(6, 2), (7, 1), (16, 4), (32, 2)])
def test_plain_padded_vs_oracle(N, pad):
    from phaser_b200.core import SpatialCorrelation
    rng = np.random.default_rng(N * 7 + pad)
    f = rng.standard_normal((1, N ** 3))
    g = rng.standard_normal((1, N ** 3))
    corr = SpatialCorrelation(N, pad)
    vol = corr.correlateSignals(list(f), list(g))
    ref, size = O.spatial_correlation_padded(f, g, N, pad, mode=0)
    check(vol, ref, size)


@pytest.mark.parametrize("N,pad,lo,hi", [(8, 1, 1, 6), (9, 2, 0, 5), (16, 3, 2, 12)])
def test_lowpass_padded_vs_oracle(N, pad, lo, hi):
    from phaser_b200.core import SpatialCorrelationLowPass
    rng = np.random.default_rng(N + pad + lo + hi)
    f = rng.standard_normal((2, N ** 3))
    g = rng.standard_normal((2, N ** 3))
    corr = SpatialCorrelationLowPass(N, pad, lower=lo, upper=hi)
    vol = corr.correlateSignals(list(f), list(g))
    ref, size = O.spatial_correlation_padded(f, g, N, pad, mode=2, lower=lo, upper=hi)
    check(vol, ref, size)


def test_laplace_state_across_calls():
    # the same object twice: the second call's first channel reads the tail
    # the first call's last channel left (and a zero last channel leaves none)
    from phaser_b200.core import SpatialCorrelationLaplace
    N, pad = 10, 2
    rng = np.random.default_rng(3)
    calls = [(rng.standard_normal((4, N ** 3)), rng.standard_normal((4, N ** 3))) for _ in range(3)]
    calls[1][0][3] = 0
    calls[1][1][3] = 0
    corr = SpatialCorrelationLaplace(N, pad)
    st = O.new_padded_state(N)
    for f, g in calls:
        vol = corr.correlateSignals(list(f), list(g))
        ref, size = O.spatial_correlation_padded(f, g, N, pad, mode=1, state=st)
        check(vol, ref, size)


def test_padded_registration_decodes_on_padded_grid():
    """register_pair with padding: the translation voxel is the argmax of the
    padded correlation of the discretised clouds (oracle), and decodes with
    N + 2 pad voxels per axis (PhaseAligner::getNumberOfVoxels)."""
    from phaser_b200 import native as nat, scene
    w = scene.WORKLOADS[0]
    pair = scene.workload_pair(0, 0)
    pad = 3
    c = nat.Context(spherical_bandwidth=w["bw"], spatial_n_voxels=w["n_voxels"], spatial_discretize_lower=w["lo"],
                    spatial_discretize_upper=w["hi"], spatial_zero_padding=pad, flags=nat.PHGPU_FLAG_KEEP_VOLUMES)
    pose = c.register_pair((pair.target.xyzi, None), (pair.source.xyzi, None))
    vol = c.spatial_result(volume=True)[2]
    c.close()
    N, M = w["n_voxels"], w["n_voxels"] + 2 * pad
    T = O.rotation_xyz(*pose.xyz)
    f = O.discretize(pair.target.xyzi, None, None, N, w["lo"], w["hi"])
    g = O.discretize(O.transform(pair.source.xyzi, T), None, None, N, w["lo"], w["hi"])
    ref, size = O.spatial_correlation_padded(f, g, N, pad, mode=1)
    check(vol, ref, size)
    vox = int(np.argmax(ref[:size]))
    if distinct_max(ref[:size]):
        assert pose.voxel == vox
    xyz = ((pose.voxel // M) % M, pose.voxel % M, pose.voxel // (M * M))
    want = [O.translation_from_index(float(v), M, w["lo"], w["hi"]) for v in xyz]
    np.testing.assert_allclose(list(pose.trans), want, atol=1e-12)


def test_padding_not_served():
    from phaser_b200 import native as nat, scene
    pair = scene.workload_pair(0, 0)
    srv = nat.Server(max_wave=1, lanes=1, device=0)
    p = nat.default_params(spherical_bandwidth=8, spatial_n_voxels=16, spatial_zero_padding=2)
    with pytest.raises(nat.PhgpuError):
        srv.submit(p, (pair.target.xyzi, None), (pair.source.xyzi, None))
    srv.close()
