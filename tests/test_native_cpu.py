"""CPU-side checks of the C ABI library: it loads without a GPU, exports every
symbol the header declares, and its host-side pose arithmetic equals the
oracle's restatement of the reference.  No device compute is called."""
import os
import re

import numpy as np
import pytest

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_symbols():
    txt = open(os.path.join(ROOT, "include", "phaser_gpu.h")).read()
    return sorted(set(re.findall(r"\b(phgpu_[a-z0-9_]+)\s*\(", txt)))


@pytest.fixture(scope="module")
def native():
    from phaser_b200 import build, native
    if not os.path.exists(native.LIB_PATH):
        build.build()
    native.load()
    return native


def test_library_exports_every_declared_symbol(native):
    import ctypes
    lib = ctypes.CDLL(native.LIB_PATH)
    syms = _header_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(lib, s)]
    assert missing == []
    assert sorted(native.EXPORTED) == syms


def test_params_default_match_reference_flags(native):
    p = native.default_params()
    # phaser_common/src/common/core-gflags.cc:6-40
    assert p.spherical_bandwidth == 75
    assert p.spherical_zero_padding == 0
    assert p.spatial_n_voxels == 100
    assert p.spatial_discretize_lower == -50 and p.spatial_discretize_upper == 50
    assert p.spatial_low_pass_lower == 0 and p.spatial_low_pass_upper == 100000
    assert p.n_channels == 4 and p.fusion_levels == 5


@pytest.mark.parametrize("bw", [8, 32, 100, 150])
def test_pose_from_bin_matches_oracle(native, bw):
    rng = np.random.default_rng(bw)
    for b in rng.integers(0, 8 * bw ** 3, size=50):
        zyz, q, xyz, T = native.pose_from_bin(int(b), bw)
        ozyz, oq, oxyz = O.bin_to_pose(int(b), bw)
        assert np.array_equal(zyz, ozyz)
        assert np.array_equal(xyz, oxyz)
        np.testing.assert_array_equal(T, O.rotation_xyz(*[np.float32(v) for v in xyz]))


def test_translation_from_index_matches_oracle(native):
    for idx in [0, 1, 50, 99, 100, 101, 150, 199]:
        for lo, hi in [(-10, 10), (-50, 50), (0, 3)]:
            assert native.translation_from_index(idx, 200, lo, hi) == O.translation_from_index(idx, 200, lo, hi)


def test_product_fails_loudly_without_library(tmp_path):
    from phaser_b200 import native
    saved = native._LIB
    native._LIB = None
    try:
        with pytest.raises(native.PhgpuError):
            native.load(str(tmp_path / "missing.so"))
    finally:
        native._LIB = saved


def test_context_creation_without_gpu_raises(native):
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(native.PhgpuError):
        native.Context(spherical_bandwidth=8, spatial_n_voxels=8)


def test_make_cloud_rejects_bad_host_inputs(native):
    # arrays the C ABI would read out of bounds are refused before the call
    good = np.zeros((10, 4), np.float32)
    c, _ = native.make_cloud(good)
    assert c.n_points == 10 and c.on_device == 0
    with pytest.raises(ValueError):
        native.make_cloud(np.zeros((10, 3), np.float32))
    with pytest.raises(ValueError):
        native.make_cloud(good, reflectivity=np.zeros(9, np.float32))
    with pytest.raises(ValueError):
        native.make_cloud(good, ambient=np.zeros((10, 2), np.float32))


def test_noalloc_wrapper_rejects_host_cloud(native):
    import torch
    p = native.default_params(spherical_bandwidth=8)
    with pytest.raises(ValueError):
        native.sample_s2_noalloc(p, torch.zeros(10, 4), None, None, torch.zeros(4 * 256))


def test_tuning_cache_round_trip(native, tmp_path):
    from phaser_b200 import tuning
    p = native.default_params(spherical_bandwidth=100, spatial_n_voxels=200, precision=1)
    path = str(tmp_path / "t.json")
    assert tuning.load(p, "B200", path) is None
    tuning.save(p, "B200", {"fuse_z_tile": 4, "so3_beta_tile": 16, "tc_chunk": 32, "radix_order": 0}, 0.5, path)
    hit = tuning.load(p, "B200", path)
    assert hit["tuning"]["fuse_z_tile"] == 4 and hit["ms_per_pair"] == 0.5
    assert tuning.load(p, "other", path) is None
    p2 = native.default_params(spherical_bandwidth=100, spatial_n_voxels=200, precision=0)
    assert tuning.load(p2, "B200", path) is None


def test_tuning_cache_is_per_build(native, tmp_path):
    """Parameters tuned under one library build are not reused by another."""
    from phaser_b200 import tuning
    p = native.default_params(spherical_bandwidth=100, spatial_n_voxels=200, precision=1)
    path = str(tmp_path / "t.json")
    b = native.build_id()
    assert len(b) == 12 and int(b, 16) >= 0 and native.build_id() == b
    tuning.save(p, "B200", {"fuse_z_tile": 8}, 0.4, path, build=b)
    assert tuning.load(p, "B200", path, build=b)["tuning"]["fuse_z_tile"] == 8
    assert tuning.load(p, "B200", path, build="0" * 12) is None
    assert tuning.load(p, "B200", path) is None
