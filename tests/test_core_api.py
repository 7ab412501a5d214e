"""The Python mirror of the reference classes (phaser_b200.core), exercised the
way the reference's own tests exercise the C++ classes."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_spatial_correlation_end_to_end():
    # phaser_core/test/translation-alignment/spatial-correlation-test.cc:59-79
    from phaser_b200.core import SpatialCorrelation
    f = np.zeros(27)
    g = np.zeros(27)
    f[0] = 1
    g[1] = 1
    corr = SpatialCorrelation(3)
    c = corr.correlateSignals([f], [g])
    assert list(O.ind2sub(int(np.argmax(c)), 3, 3)) == [0, 2, 0]


def test_spatial_correlation_random_nonzero():
    # spatial-correlation-test.cc:42-57
    from phaser_b200.core import SpatialCorrelation
    rng = np.random.default_rng(0)
    corr = SpatialCorrelation(3)
    c = corr.correlateSignals([rng.uniform(0, 100, 27)], [rng.uniform(0, 100, 27)])
    assert np.count_nonzero(c) > 0


def test_spherical_laplace_mirror_matches_oracle():
    from phaser_b200.core import SphericalCorrelationLaplace
    bw = 10
    rng = np.random.default_rng(3)
    f = [rng.standard_normal(4 * bw * bw) for _ in range(4)]
    g = [rng.standard_normal(4 * bw * bw) for _ in range(4)]
    corr = SphericalCorrelationLaplace(bw)
    corr.correlateSampledSignals(f, g)
    vol = corr.getCorrelation()
    ref = O.spherical_correlation(np.array(f), np.array(g), bw)
    assert int(np.argmax(vol)) == O.argmax(ref)
    assert corr.getBandwidth() == bw
    with pytest.raises(ValueError):
        corr.correlateSampledSignals(f[:1], g[:1])


def test_registration_and_aligner_mirror():
    from phaser_b200 import scene
    from phaser_b200.core import PhaseAligner, SphOptRegistration
    w = scene.WORKLOADS[0]
    p = scene.workload_pair(0, 1)
    reg = SphOptRegistration(bandwidth=w["bw"], n_voxels=w["n_voxels"], lower=w["lo"], upper=w["hi"])
    pose = reg.registerPointCloud((p.target.xyzi, None), (p.source.xyzi, None))
    ref = O.register_pair(p.target.xyzi, None, p.source.xyzi, None, w["bw"], w["n_voxels"], w["lo"], w["hi"])
    assert (pose["rot_bin"], pose["voxel"]) == (ref.rot_bin, ref.voxel)
    al = PhaseAligner(w["n_voxels"], w["lo"], w["hi"])
    al.alignRegistered((p.target.xyzi, None), (p.source.xyzi, None))
    c = al.getCorrelation()
    assert c.shape == (w["n_voxels"] ** 3,)
    assert al.getNumberOfVoxels() == w["n_voxels"]
