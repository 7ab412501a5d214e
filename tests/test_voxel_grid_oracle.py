"""The oracle's voxel-grid restatement (orc_voxel_grid) pinned against an
independent numpy restatement of pcl::VoxelGrid<PointXYZI>::applyFilter
(PCL 1.8.1, used by phaser_pre/src/commands/voxel-grid-cmd.cc:11-22; PCL is
not in the reference tree, so its published algorithm is restated twice) and
against the reference's own VoxelGridCmdTest
(phaser_pre/test/cloud-pre-processor-test.cc:54-64: 500 points uniform in
[0, pi)^3 lose points under the 0.25 leaf).  Both restatements sum a leaf's
points in input order in float32, so they agree bit for bit."""
import numpy as np
import pytest

from oracle import oracle as O


def np_voxel_grid(xyzi, leaf=0.25, min_points=0, refl=None):
    x = np.asarray(xyzi, np.float32)
    fin = np.isfinite(x[:, :3]).all(axis=1)
    pts, idx = x[fin], np.nonzero(fin)[0]
    if len(pts) == 0:
        return np.zeros((0, 4), np.float32), None
    inv = np.float32(1) / np.broadcast_to(np.asarray(leaf, np.float32), (3,))
    mn, mx = pts[:, :3].min(axis=0), pts[:, :3].max(axis=0)
    d = ((mx - mn) * inv).astype(np.int64) + 1
    if d[0] * d[1] * d[2] > 2 ** 31 - 1:
        return x.copy(), None if refl is None else np.asarray(refl, np.float32).copy()
    min_b = np.floor(mn * inv).astype(np.int64)
    div = np.floor(mx * inv).astype(np.int64) - min_b + 1
    ijk = (np.floor(pts[:, :3] * inv) - min_b.astype(np.float32)).astype(np.int64)
    key = ijk[:, 0] + ijk[:, 1] * div[0] + ijk[:, 2] * div[0] * div[1]
    order = np.argsort(key, kind="stable")
    skey = key[order]
    starts = np.nonzero(np.r_[True, skey[1:] != skey[:-1]])[0]
    ends = np.r_[starts[1:], len(skey)]
    counts = ends - starts
    keep = counts >= min_points
    starts, counts = starts[keep], counts[keep]
    vals = pts[order]
    rv = None if refl is None else np.asarray(refl, np.float32)[idx][order]
    acc = np.zeros((len(starts), 4), np.float32)
    racc = np.zeros(len(starts), np.float32)
    for j in range(int(counts.max()) if len(counts) else 0):  # j-th point of every leaf: sequential float32 sums
        live = counts > j
        acc[live] = acc[live] + vals[starts[live] + j]
        if rv is not None:
            racc[live] = racc[live] + rv[starts[live] + j]
    c = counts.astype(np.float32)
    return acc / c[:, None], None if rv is None else racc / c


def lidar_like(n, seed, scale=30.0):
    rng = np.random.default_rng(seed)
    ang = rng.uniform(0, 2 * np.pi, n)
    r = rng.gamma(2.0, scale / 4, n)
    z = rng.normal(0, 2, n)
    return np.stack([r * np.cos(ang), r * np.sin(ang), z, rng.uniform(0, 1000, n)], axis=1).astype(np.float32)


def check(xyzi, leaf=0.25, min_points=0, refl=None):
    got = O.voxel_grid(xyzi, leaf, min_points, refl)
    want, wrefl = np_voxel_grid(xyzi, leaf, min_points, refl)
    assert got is not None
    assert got[0].shape == want.shape
    assert np.array_equal(got[0], want, equal_nan=True)
    if refl is not None:
        assert np.array_equal(got[1], wrefl)
    return got


def test_reference_voxel_grid_cmd_case():
    # VoxelGridCmdTest: 500 random points in [0, pi)^3 -> fewer points
    rng = np.random.default_rng(54)
    x = rng.uniform(0, np.pi, (500, 4)).astype(np.float32)
    out = check(x)[0]
    assert len(out) < 500
    # centroids stay inside the sampled box
    assert (out[:, :3] >= 0).all() and (out[:, :3] < np.float32(np.pi)).all()


@pytest.mark.parametrize("n,seed,leaf,minp", [(5000, 1, 0.25, 0), (20000, 2, 0.5, 0), (20000, 3, 0.1, 3),
                                              (3000, 4, (0.2, 0.3, 0.7), 0), (1, 5, 0.25, 0), (7, 6, 10.0, 2)])
def test_oracle_matches_numpy(n, seed, leaf, minp):
    x = lidar_like(n, seed)
    refl = np.random.default_rng(seed + 100).uniform(0, 255, n).astype(np.float32)
    check(x, leaf, minp, refl)


def test_negative_and_boundary_coordinates():
    # points exactly on leaf boundaries and negative coordinates
    g = np.arange(-8, 8, dtype=np.float32) * np.float32(0.25)
    xx, yy, zz = np.meshgrid(g, g, g, indexing="ij")
    x = np.stack([xx.ravel(), yy.ravel(), zz.ravel(), np.arange(xx.size, dtype=np.float32)], axis=1)
    out = check(np.concatenate([x, x + np.float32(0.1)]))[0]
    assert len(out) == 16 ** 3


def test_non_finite_points_dropped():
    x = lidar_like(4000, 7)
    x[::13, 0] = np.nan
    x[5::17, 2] = np.inf
    out = check(x)[0]
    assert np.isfinite(out).all()


def test_overflow_returns_input():
    # dx*dy*dz > INT32_MAX: PCL warns and returns the input unchanged
    x = lidar_like(1000, 8, scale=500.0)
    out = O.voxel_grid(x, 1e-3)
    assert np.array_equal(out[0], x)


def test_range_refused_and_empty():
    x = lidar_like(100, 9) + np.float32(3e9)
    x[:, 3] = 1
    assert O.voxel_grid(x, 0.25) is None
    assert len(O.voxel_grid(np.zeros((0, 4), np.float32), 0.25)[0]) == 0
    nanc = np.full((10, 4), np.nan, np.float32)
    assert len(O.voxel_grid(nanc, 0.25)[0]) == 0
