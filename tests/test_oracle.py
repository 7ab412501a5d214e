"""CPU tests of the oracle: golden vectors from the reference's own tests and
fixtures produced by the reference's SOFT sources (tests/golden)."""
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden", "soft_reference_small.npz")


def test_sub2ind_golden():
    # phaser_common/test/utils/signal-utils-test.cc:210-215
    assert O.sub2ind(100, 100, 100, 201, 201) == 4060300
    assert O.sub2ind(120, 120, 120, 201, 201) == 4872360
    assert O.sub2ind(80, 80, 80, 201, 201) == 3248240
    for lin in (0, 1, 4060300, 201 ** 3 - 1):
        x, y, z = O.ind2sub(lin, 201, 201)
        assert O.sub2ind(x, y, z, 201, 201) == lin


def test_pyramid_struct_golden():
    # phaser_core/test/fusion/pyramid-struct-test.cc:21-33
    lb, ub, co = O.pyramid_struct(100, 2)
    assert list(co) == [50, 25]
    assert list(lb) == [25, 13]
    assert list(ub) == [75, 38]


@pytest.mark.parametrize("n", [8, 9, 100, 101])
def test_fftshift_round_trip(n):
    # phaser_common/test/utils/signal-utils-test.cc:32-208
    x = np.arange(n) + 1j * np.arange(n)[::-1]
    s = O.fftshift(x)
    assert np.allclose(O.ifftshift(s), x)
    assert np.allclose(s, np.fft.fftshift(x))


@pytest.mark.parametrize("n", [3, 8, 64, 200, 134, 67, 512])
def test_fft_against_definition(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    a = x.copy().view(np.float64).copy()
    O.lib().orc_fft1d(a, n, -1)
    np.testing.assert_allclose(a.view(np.complex128), np.fft.fft(x), atol=1e-11 * n)


def test_spatial_delta_known_answer():
    # phaser_core/test/translation-alignment/spatial-correlation-test.cc:59-79
    f = np.zeros(27)
    g = np.zeros(27)
    f[0] = 1
    g[1] = 1
    c = O.spatial_correlation(f[None], g[None], 3, laplace=False)
    assert list(O.ind2sub(O.argmax(c), 3, 3)) == [0, 2, 0]


@pytest.mark.parametrize("n", [27, 48, 50, 100, 320, 998, 1024])
def test_positional_fusion_equals_literal_pyramid(n):
    rng = np.random.default_rng(n)
    ch = rng.standard_normal((4, n)) + 1j * rng.standard_normal((4, n))
    lit = O.fuse_literal(ch)
    pos = np.zeros(n, complex)
    for p in range(n):
        r = O.fusion_rule(p, n)
        if r == 1:
            pos[p] = 0
        elif r == 2:
            pos[p] = ch[:, p].sum() / 4
        else:
            pos[p] = ch[int(np.argmax(np.abs(ch[:, p]) ** 2)), p]
    np.testing.assert_allclose(lit, pos, atol=1e-15)


def test_fusion_band_quirk_zero_slot():
    # n/4 with fraction .5: PyramidStruct keeps one more coefficient than
    # expand() restores, leaving a zero at the first expand upper bound.
    n = 50  # 50/4 = 12.5 -> lb 13, struct ub 38, expand ub 37
    assert O.fusion_rule(37, n, levels=1) == 1
    assert O.fusion_rule(36, n, levels=1) == 2
    assert O.fusion_rule(12, n, levels=1) == 0


def test_oracle_sht_matches_soft_fixture():
    d = np.load(GOLD)
    c = O.sht(d["sht_b8_signal"], 8)
    np.testing.assert_allclose(c, d["sht_b8_coef"], atol=1e-13)


def test_oracle_laplace_sph_matches_soft_fixture():
    d = np.load(GOLD)
    corr = O.spherical_correlation(d["sph_b8_f"], d["sph_b8_g"], 8)
    ref = d["sph_b8_corr"]
    assert np.abs(corr - ref).max() <= 1e-12 * np.abs(ref).max()
    assert O.argmax(corr) == int(d["sph_b8_argmax"])


def test_oracle_single_channel_padded_matches_soft_fixture():
    d = np.load(GOLD)
    corr = O.spherical_correlation(d["sph1_b6p2_f"], d["sph1_b6p2_g"], 6, 8)
    ref = d["sph1_b6p2_corr"]
    assert np.abs(corr - ref).max() <= 1e-12 * np.abs(ref).max()


def test_oracle_spatial_matches_fixture():
    d = np.load(GOLD)
    c = O.spatial_correlation(d["spat_n6_f"], d["spat_n6_g"], 6, laplace=True)
    np.testing.assert_allclose(c, d["spat_n6_c"], atol=1e-12 * np.abs(d["spat_n6_c"]).max())


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("bw,C", [(4, 1), (8, 4), (12, 3), (16, 4)])
def test_oracle_vs_soft_live(bw, C):
    rng = np.random.default_rng(bw * 10 + C)
    f = rng.standard_normal((C, 4 * bw * bw))
    g = rng.standard_normal((C, 4 * bw * bw))
    a = O.spherical_correlation(f, g, bw)
    b = O.ref_spherical_correlation(f, g, bw)
    assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()
    assert O.argmax(a) == O.argmax(b)


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("N,C,lap", [(3, 1, False), (4, 4, True), (7, 3, True), (8, 4, True)])
def test_oracle_vs_reference_spatial_buffers(N, C, lap):
    # the literal restatement keeps the reference's N^3-long half-spectrum
    # buffers with their stale tail; the oracle works on the valid region only
    rng = np.random.default_rng(N)
    f = rng.standard_normal((C, N ** 3))
    g = rng.standard_normal((C, N ** 3))
    a = O.spatial_correlation(f, g, N, laplace=lap)
    b = O.ref_spatial_correlation(f, g, N, laplace=lap)
    np.testing.assert_allclose(a, b, atol=1e-12 * np.abs(b).max())


def test_wigner_orthonormality():
    # int_0^pi d^l d^l' sin(beta) = delta with the Driscoll-Healy weights
    bw = 10
    w = O.dh_weights(bw)
    betas = np.pi * (2 * np.arange(2 * bw) + 1) / (4 * bw)
    for m1, m2 in [(0, 0), (2, -3), (-4, 1), (5, 5), (-6, -2)]:
        j0 = max(abs(m1), abs(m2))
        D = np.array([O.wigner_column(m1, m2, bw, b) for b in betas])  # [k, l]
        G = (D * w[:, None]).T @ D
        np.testing.assert_allclose(G, np.eye(bw - j0), atol=1e-12)


def test_histc_edges_and_aliasing():
    N, lo, hi = 4, -2, 2
    e = O.edges(N, lo, hi)
    assert e[0] == np.float32(-2) and e[-1] == np.float32(2)
    pts = np.array([[0.1, 0.1, 0.1, 1.0],      # inside
                    [2.0, 2.0, 2.0, 1.0],      # on last edge -> bin N-1
                    [-3.0, 0.1, 0.1, 1.0],     # x out of range -> aliases
                    [0.1, 0.1, -3.0, 1.0]],    # z out of range -> skipped
                   np.float32)
    lin = O.voxel_index(pts, N, lo, hi)
    b = [int(np.searchsorted(e, 0.1, side="right") - 1)] * 3
    assert lin[0] == b[0] * N + b[1] + N * N * b[2]
    assert lin[1] == (N - 1) * N + (N - 1) + N * N * (N - 1)
    assert lin[2] == (((0xFFFFFFFF * N) + b[1] + N * N * b[2]) & 0xFFFFFFFF)
    assert lin[3] == 0xFFFFFFFF


@pytest.mark.parametrize("N,lo,hi", [(200, -10, 10), (64, -50, 40), (7, -3, 1), (101, 5, -7), (13, 0, 3)])
def test_edges_follow_eigen_linspaced(N, lo, hi):
    # Eigen >= 3.3 LinSpaced (float): counted down from hi when |hi| < |lo|
    # (e[0] = lo, e[i] = hi - (N - 1 - i) step), up from lo otherwise
    # (e[N - 1] = hi); step = (hi - lo) / (N - 1) in float
    e = O.edges(N, lo, hi)
    f32 = np.float32
    step = (f32(hi) - f32(lo)) / f32(N - 1)
    if abs(hi) < abs(lo):
        want = [f32(lo)] + [f32(hi) - f32(N - 1 - i) * step for i in range(1, N)]
    else:
        want = [f32(lo) + f32(i) * step for i in range(N - 1)] + [f32(hi)]
    np.testing.assert_array_equal(e, np.array(want, np.float32))
    assert e[0] == f32(lo) and e[-1] == f32(hi)


def test_translation_from_index():
    # translation-utils.cc:40-52, width = |lo| + |hi| + 1
    assert O.translation_from_index(0, 200, -10, 10) == 0.0
    assert O.translation_from_index(5, 200, -10, 10) == pytest.approx(5 * 21 / 200)
    assert O.translation_from_index(150, 200, -10, 10) == pytest.approx(-50 * 21 / 200)


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("sph_mode", [0, 1])
def test_oracle_registration_equals_reference_path(sph_mode):
    # SphOptRegistration (mode 0) and SphRegistration's single 0.6 I + 0.4 R
    # signal (mode 1): the FP64 restatement and the reference's SOFT sources
    # driven by the restated glue give the same bin, voxel and pose
    from phaser_b200 import scene
    pair = scene.make_pair(0, 9, beams=16, cols=256)
    args = (pair.target.xyzi, pair.target.reflectivity, pair.source.xyzi, pair.source.reflectivity, 8, 16, -10, 10)
    rb, vx, pose6 = O.ref_register_pair(*args, threads=2, sph_mode=sph_mode)
    pose = O.register_pair(*args, sph_mode=sph_mode)
    assert (pose.rot_bin, pose.voxel) == (rb, vx)
    assert list(pose.xyz) == list(pose6[:3]) and list(pose.trans) == list(pose6[3:])


def test_mix_signal_is_the_reference_weighting():
    # retrieveInterpolation (spherical-correlation.cc:103-112)
    s = np.arange(8, dtype=np.float64).reshape(2, 4)  # channels {range, intensity}, 4 directions
    out = np.zeros(4)
    O.lib().orc_mix_signal(s.reshape(-1).ctypes.data, 4, out.ctypes.data)
    np.testing.assert_array_equal(out, 0.6 * s[1] + 0.4 * s[0])
