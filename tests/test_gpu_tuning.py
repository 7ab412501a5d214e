"""Autotuner (phgpu_autotune): every candidate of the tile and chunk
parameters gives bit-identical volumes; the radix orders of runtime FFT plans
keep the results within the FP32 parity bar of the FP64 oracle; the search
returns valid parameters and the context keeps them."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nat():
    from phaser_b200 import native
    native.load()
    return native


def _volumes(c, clouds):
    pose = c.register_pair(*clouds)
    _, _, rv = c.sph_result(volume=True)
    _, _, tv = c.spatial_result(volume=True)
    return pose, rv, tv


@pytest.mark.parametrize("precision", [0, 1])
def test_tile_parameters_do_not_change_results(nat, precision):
    from phaser_b200 import scene
    w = scene.WORKLOADS[1]
    pair = scene.workload_pair(1, 1)
    clouds = ((pair.target.xyzi, pair.target.reflectivity), (pair.source.xyzi, pair.source.reflectivity))
    c = nat.Context(spherical_bandwidth=w["bw"], spatial_n_voxels=w["n_voxels"], spatial_discretize_lower=w["lo"],
                    spatial_discretize_upper=w["hi"], flags=nat.PHGPU_FLAG_KEEP_VOLUMES, precision=precision)
    p0, r0, t0 = _volumes(c, clouds)
    trials = [{"fuse_z_tile": f} for f in (2, 4, 8)] + [{"so3_beta_tile": b} for b in (8, 32)]
    if precision:
        trials += [{"tc_chunk": 16}, {"tc_chunk": 32}]
    for t in trials:
        c.set_tuning(dict({"fuse_z_tile": 0, "so3_beta_tile": 0, "tc_chunk": 0, "radix_order": 0}, **t))
        p1, r1, t1 = _volumes(c, clouds)
        assert (p1.rot_bin, p1.voxel) == (p0.rot_bin, p0.voxel), t
        # the voxel sums are float atomics (their order varies): translation volumes within 1e-6
        assert np.array_equal(r1, r0), t
        assert np.linalg.norm(t1 - t0) <= 1e-6 * np.linalg.norm(t0), t
    best, ms = c.autotune(*clouds, reps=2)
    assert ms > 0 and c.tuning() == best
    print(f"precision {precision}: best {best}, {ms:.3f} ms per registration")
    with pytest.raises(nat.PhgpuError):
        c.set_tuning({"so3_beta_tile": 7})


@pytest.mark.parametrize("order", [0, 1, 2])
def test_radix_orders_keep_parity(nat, order):
    # the run script's translation grid (N = 201 = 3 * 67, runtime plans) and
    # an S^2 / SO(3) length on runtime plans (2B = 48)
    from phaser_b200 import scene
    pair = scene.workload_pair(0, 0)
    bw, N, lo, hi = 24, 201, -50, 50
    c = nat.Context(spherical_bandwidth=bw, spatial_n_voxels=N, spatial_discretize_lower=lo,
                    spatial_discretize_upper=hi, flags=nat.PHGPU_FLAG_KEEP_VOLUMES)
    c.set_tuning({"radix_order": order})
    pose, rv, tv = _volumes(c, ((pair.target.xyzi, None), (pair.source.xyzi, None)))
    res = O.register_pair(pair.target.xyzi, None, pair.source.xyzi, None, bw, N, lo, hi, want_volumes=True)
    assert (pose.rot_bin, pose.voxel) == (res[0].rot_bin, res[0].voxel)
    assert np.linalg.norm(rv - res[1]) <= 1e-5 * np.linalg.norm(res[1])
    assert np.linalg.norm(tv - res[2]) <= 1e-5 * np.linalg.norm(res[2])
