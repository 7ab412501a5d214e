"""Tensor-core contractions (PHGPU_PRECISION_TF32X3 / BF16X3: the Legendre sums
of the forward SHT and the Wigner-d sums of the SO(3) synthesis, both on
tcgen05) against the FP64 oracle and the FP32 CUDA-core path.  The volume
error bounds the error of both contractions, the correlation being linear in
each side's coefficients.

Bar: identical rotation bins and a correlation-volume relative L2 error of at
most 1e-5 against the FP64 oracle at the B = 100 workload and, for tf32x3, in
every case.  bf16x3 operands carry 16 to 17 significant bits (hi = bf16(x),
lo = bf16(x - hi)): on random signals its error floor is 7-8e-6, and on the
smallest case (one 8 x 8 signal, whose few products do not average) 1.0e-5
was measured, so the small random cases hold it to 1.5e-5.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

REL_L2 = 1e-5
REL_L2_SMALL = {"tf32x3": 1e-5, "bf16x3": 1.5e-5}
PRECISIONS = {"tf32x3": 1, "bf16x3": 2}


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def nat():
    from phaser_b200 import native
    native.load()
    return native


@pytest.mark.parametrize("prec", sorted(PRECISIONS))
@pytest.mark.parametrize("bw,pad,C", [(4, 0, 1), (8, 0, 4), (8, 2, 4), (16, 3, 4), (25, 0, 3), (32, 0, 4),
                                      (64, 0, 4), (8, 152, 2)])
def test_tc_spherical_vs_oracle(nat, prec, bw, pad, C):
    rng = np.random.default_rng(bw * 100 + pad * 10 + C)
    f = rng.standard_normal((C, 4 * bw * bw))
    g = rng.standard_normal((C, 4 * bw * bw))
    c = nat.Context(spherical_bandwidth=bw, spherical_zero_padding=pad, spatial_n_voxels=4,
                    flags=nat.PHGPU_FLAG_KEEP_VOLUMES, precision=PRECISIONS[prec])
    c.sph_correlate(list(f), list(g))
    b, _, vol = c.sph_result(volume=True)
    ref = O.spherical_correlation(f, g, bw, bw + pad)
    err = rel_l2(vol, ref)
    print(f"{prec} bw={bw} pad={pad} C={C}: rel_l2 {err:.3e}")
    assert err <= REL_L2_SMALL[prec]
    assert b == O.argmax(ref)


@pytest.mark.parametrize("prec", sorted(PRECISIONS))
def test_tc_register_pair_full_size(nat, prec):
    # B = 100, N = 200 bench workload: tensor-core and FP32 contexts agree on
    # the pose, and the rotation volume stays within 1e-5 of the FP64 oracle
    from phaser_b200 import scene
    w = scene.WORKLOADS[1]
    pair = scene.workload_pair(1, 0)
    args = ((pair.target.xyzi, pair.target.reflectivity), (pair.source.xyzi, pair.source.reflectivity))
    kw = dict(spherical_bandwidth=w["bw"], spatial_n_voxels=w["n_voxels"], spatial_discretize_lower=w["lo"],
              spatial_discretize_upper=w["hi"], flags=nat.PHGPU_FLAG_KEEP_VOLUMES)
    ref_ctx = nat.Context(**kw)
    p32 = ref_ctx.register_pair(*args)
    _, _, v32 = ref_ctx.sph_result(volume=True)
    tc = nat.Context(precision=PRECISIONS[prec], **kw)
    ptc = tc.register_pair(*args)
    _, _, vtc = tc.sph_result(volume=True)
    f, _ = ref_ctx.samples(0)
    g, _ = ref_ctx.samples(1)
    ref = O.spherical_correlation(f, g, w["bw"], w["bw"])
    e_tc, e_32 = rel_l2(vtc, ref), rel_l2(v32, ref)
    print(f"{prec} B=100 pair: rel_l2 tensor {e_tc:.3e}, fp32 {e_32:.3e}")
    assert (ptc.rot_bin, ptc.voxel) == (p32.rot_bin, p32.voxel)
    assert e_tc <= REL_L2
