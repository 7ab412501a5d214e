"""End-to-end parity with the reference path: the reference's own SOFT 2.0
sources (compiled unmodified, on the project's FP64 FFTW-API shim) driven by
the restated phaser_core glue (oracle/ref_glue.c: kd-tree sampling,
SphericalCorrelationLaplace, PhaseAligner with the N^3 half-spectrum buffers)
register the same clouds as phgpu_register_pair; the rotation bin, the
translation voxel and the pose must be identical
(SphOptRegistration::registerPointCloud, sph-opt-registration.cc:34-132).

The margin between the largest and the second largest correlation value of
each GPU volume is printed: a bin or voxel could only differ where the two
top values are closer than the FP32 error of the volume.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nat():
    from phaser_b200 import native
    native.load()
    return native


def top2_margin(vol):
    v = np.asarray(vol, np.float64)
    i = int(np.argmax(v))
    top = v[i]
    v2 = np.delete(v, i).max()
    return (top - v2) / abs(top)


CASES = [(0, 0, 0, 0), (0, 1, 0, 0), (0, 2, 0, 0), (0, 3, 0, 0), (1, 0, 0, 0),  # SphOptRegistration, FP32
         (0, 0, 1, 0), (1, 0, 1, 0),                                            # tensor-core (tf32x3) synthesis
         (0, 0, 0, 1), (0, 1, 0, 1), (1, 0, 0, 1)]                              # SphRegistration's single signal


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("cfg,k,precision,sph_mode", CASES)
def test_register_pair_equals_reference_path(nat, cfg, k, precision, sph_mode):
    from phaser_b200 import scene
    w = scene.WORKLOADS[cfg]
    pair = scene.workload_pair(cfg, k)
    rb, vx, pose6 = O.ref_register_pair(pair.target.xyzi, pair.target.reflectivity, pair.source.xyzi,
                                        pair.source.reflectivity, w["bw"], w["n_voxels"], w["lo"], w["hi"],
                                        threads=12, sph_mode=sph_mode)
    c = nat.Context(spherical_bandwidth=w["bw"], spatial_n_voxels=w["n_voxels"], spatial_discretize_lower=w["lo"],
                    spatial_discretize_upper=w["hi"], flags=nat.PHGPU_FLAG_KEEP_VOLUMES, precision=precision,
                    spherical_fusion=nat.PHGPU_FUSION_MIX if sph_mode else nat.PHGPU_FUSION_LAPLACE)
    pose = c.register_pair((pair.target.xyzi, pair.target.reflectivity),
                           (pair.source.xyzi, pair.source.reflectivity))
    _, _, rvol = c.sph_result(volume=True)
    _, _, tvol = c.spatial_result(volume=True)
    print(f"config {cfg} pair {k} precision {precision} mode {sph_mode}: bin {pose.rot_bin} (ref {rb}) voxel {pose.voxel} "
          f"(ref {vx}); top-1/top-2 margin rotation {top2_margin(rvol):.3e}, translation {top2_margin(tvol):.3e}")
    assert pose.rot_bin == rb
    assert pose.voxel == vx
    assert list(pose.xyz) == list(pose6[:3])
    assert list(pose.trans) == list(pose6[3:])
