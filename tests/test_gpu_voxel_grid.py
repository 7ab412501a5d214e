"""GPU voxel-grid downsampling (phgpu_voxel_grid_*, the VoxelGridCmd
replacement) against the oracle's float32 restatement of pcl::VoxelGrid:
bit-exact centroids, counts and leaf order (both sum a leaf's points in input
order), plus the reference's own VoxelGridCmdTest property and an ingest
pipeline PLY -> pinned host -> GPU downsample -> registration."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def vg():
    from phaser_b200 import native
    v = native.VoxelGrid(1 << 21)
    yield v
    v.close()


def lidar_like(n, seed, scale=30.0):
    rng = np.random.default_rng(seed)
    ang = rng.uniform(0, 2 * np.pi, n)
    r = rng.gamma(2.0, scale / 4, n)
    z = rng.normal(0, 2, n)
    return np.stack([r * np.cos(ang), r * np.sin(ang), z, rng.uniform(0, 1000, n)], axis=1).astype(np.float32)


def same(a, b):
    return a.shape == b.shape and np.array_equal(a, b, equal_nan=True)


def test_reference_voxel_grid_cmd_case(vg):
    rng = np.random.default_rng(54)
    x = rng.uniform(0, np.pi, (500, 4)).astype(np.float32)
    out, _, _ = vg.filter(x)
    want = O.voxel_grid(x)[0]
    assert len(out) < 500
    assert same(out, want)


@pytest.mark.parametrize("n,seed,leaf,minp", [(5000, 1, 0.25, 0), (131072, 2, 0.25, 0), (131072, 3, 0.1, 3),
                                              (60000, 4, (0.2, 0.3, 0.7), 0), (1, 5, 0.25, 0), (7, 6, 10.0, 2),
                                              (1 << 20, 7, 0.25, 0), (300000, 8, 0.05, 2)])
def test_matches_oracle(vg, n, seed, leaf, minp):
    x = lidar_like(n, seed)
    rng = np.random.default_rng(seed + 50)
    refl = rng.uniform(0, 255, n).astype(np.float32)
    amb = rng.uniform(0, 60, n).astype(np.float32)
    out, orf, oam = vg.filter(x, leaf, minp, refl, amb)
    want, wrf, wam = O.voxel_grid(x, leaf, minp, refl, amb)
    assert same(out, want)
    assert same(orf, wrf) and same(oam, wam)


def test_scan_clouds_match_oracle(vg):
    from phaser_b200 import scene
    for wl in (1, 4):
        p = scene.workload_pair(wl, 0)
        for cl in (p.target, p.source):
            out, orf, _ = vg.filter(cl.xyzi, 0.25, 0, cl.reflectivity)
            want, wrf, _ = O.voxel_grid(cl.xyzi, 0.25, 0, cl.reflectivity)
            assert same(out, want)
            if cl.reflectivity is not None:
                assert same(orf, wrf)
            assert len(out) < len(cl.xyzi)


def test_non_finite_dropped(vg):
    x = lidar_like(40000, 9)
    x[::13, 0] = np.nan
    x[5::17, 2] = np.inf
    x[7::19, 1] = -np.inf
    out, _, _ = vg.filter(x)
    assert same(out, O.voxel_grid(x)[0])
    assert np.isfinite(out).all()


def test_overflow_returns_input(vg):
    x = lidar_like(1000, 10, scale=500.0)
    r = np.arange(1000, dtype=np.float32)
    out, orf, _ = vg.filter(x, 1e-3, 0, r)
    assert same(out, x) and same(orf, r)


def test_range_refused(vg):
    from phaser_b200 import native
    x = lidar_like(100, 11) + np.float32(3e9)
    assert O.voxel_grid(x, 0.25) is None
    with pytest.raises(native.PhgpuError):
        vg.filter(x, 0.25)


def test_empty_and_degenerate(vg):
    assert len(vg.filter(np.zeros((0, 4), np.float32))[0]) == 0
    assert len(vg.filter(np.full((10, 4), np.nan, np.float32))[0]) == 0
    one = np.array([[1.0, -2.0, 3.0, 4.0]], np.float32)
    assert same(vg.filter(one)[0], one)
    same_pt = np.repeat(one, 5000, axis=0)
    assert same(vg.filter(same_pt)[0], O.voxel_grid(same_pt)[0])
    assert len(vg.filter(same_pt, 0.25, 5001)[0]) == 0


def test_device_buffers_and_reuse(vg):
    import torch
    x = lidar_like(70000, 12)
    want = O.voxel_grid(x, 0.3, 2)[0]
    xd = torch.from_numpy(x).cuda()
    out, _, _ = vg.filter(xd, 0.3, 2, out_device=True)
    assert out.is_cuda
    assert same(out.cpu().numpy(), want)
    # smaller then larger clouds through the same handle
    for n, s in ((100, 13), (200000, 14), (3000, 15)):
        y = lidar_like(n, s)
        assert same(vg.filter(y)[0], O.voxel_grid(y)[0])


def test_capacity_and_leaf_checks(vg):
    from phaser_b200 import native
    small = native.VoxelGrid(100)
    with pytest.raises(native.PhgpuError):
        small.filter(lidar_like(101, 16))
    with pytest.raises(native.PhgpuError):
        small.filter(lidar_like(10, 16), (0.25, 0.0, 0.25))
    small.close()


def test_ply_to_registration_pipeline(tmp_path):
    """PLY files -> pinned host buffers -> GPU voxel grid -> registration;
    the pose equals the oracle's on the oracle-downsampled clouds."""
    from phaser_b200 import native, scene
    from phaser_b200.core import PlyHelper, VoxelGridCmd
    w = scene.WORKLOADS[0]
    pair = scene.workload_pair(0, 0)
    paths = []
    for name, cl in (("t", pair.target), ("s", pair.source)):
        p = tmp_path / f"{name}.ply"
        head = (f"ply\nformat binary_little_endian 1.0\nelement vertex {len(cl.xyzi)}\n"
                "property float x\nproperty float y\nproperty float z\nproperty float intensity\nend_header\n")
        p.write_bytes(head.encode() + np.ascontiguousarray(cl.xyzi, "<f4").tobytes())
        paths.append(p)
    helper = PlyHelper()
    cmd = VoxelGridCmd(0.25, max_points=1 << 18)
    clouds, oclouds = [], []
    for p, cl in zip(paths, (pair.target, pair.source)):
        pc = helper.readPlyFromFile(str(p), pinned=True)
        assert np.array_equal(pc.xyzi.numpy(), cl.xyzi)
        xyzi, _, _ = cmd.execute(pc.cloud())
        oxyzi = O.voxel_grid(cl.xyzi)[0]
        assert same(xyzi, oxyzi)
        clouds.append(xyzi)
        oclouds.append(oxyzi)
    c = native.Context(spherical_bandwidth=w["bw"], spatial_n_voxels=w["n_voxels"], spatial_discretize_lower=w["lo"],
                       spatial_discretize_upper=w["hi"])
    pose = c.register_pair((clouds[0], None), (clouds[1], None))
    c.close()
    opose = O.register_pair(oclouds[0], None, oclouds[1], None, w["bw"], w["n_voxels"], w["lo"], w["hi"])
    assert (pose.rot_bin, pose.voxel) == (opose.rot_bin, opose.voxel)
