"""Precision of the SO(3) synthesis at B = 256 (the large-pair workload:
256 x 4096 LiDAR scans, ~1M points, a 512^3 SO(3) grid): the FP32 CUDA-core
synthesis, the tensor-core split-TF32 (tf32x3) and split-BF16 (bf16x3)
syntheses, each against the FP64 oracle on a subset of beta slices (the full
FP64 volume would take minutes); the subset includes the slice of the argmax.

Prints one table row per precision: relative L2 error of |z|^2 over the
slices, the rotation bin, and whether the oracle's argmax inside the bin's
slice is the same (alpha, gamma)."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

REL_L2 = 1e-5
NAMES = {0: "fp32 (CUDA cores)", 1: "tf32x3 (tensor cores)", 2: "bf16x3 (tensor cores)"}


def test_precision_table_b256():
    from phaser_b200 import native, scene
    native.load()
    bw = scene.WORKLOADS[4]["bw"]
    n = 2 * bw
    pair = scene.workload_pair(4, 0)
    cap = max(pair.target.xyzi.shape[0], pair.source.xyzi.shape[0])
    kw = dict(spherical_bandwidth=bw, spatial_n_voxels=4, max_points=cap, flags=native.PHGPU_FLAG_KEEP_VOLUMES)
    c32 = native.Context(precision=0, **kw)
    c32.sample_s2(pair.target.xyzi, pair.target.reflectivity, side=0)
    c32.sample_s2(pair.source.xyzi, pair.source.reflectivity, side=1)
    f, _ = c32.samples(0)
    g, _ = c32.samples(1)
    rows = {}
    ref = None
    ks = None
    for prec in (0, 1, 2):
        c = c32 if prec == 0 else native.Context(precision=prec, **kw)
        c.sph_correlate(list(f), list(g))
        b, _, vol = c.sph_result(volume=True)
        vol = vol.reshape(n, n, n)
        if ks is None:
            kb = b // (n * n)
            ks = sorted(set(list(range(0, n, n // 8)) + [kb]))
            ref = O.spherical_correlation_slices(f, g, bw, ks)
        v = vol[ks]
        err = float(np.linalg.norm(v - ref) / np.linalg.norm(ref))
        kb = b // (n * n)
        same = int(np.argmax(ref[ks.index(kb)])) == b % (n * n) if kb in ks else None
        rows[prec] = (err, b, same)
        del vol
        if prec:
            c.close()
    print(f"\nB={bw}: {len(ks)} beta slices {ks}")
    print("| synthesis | rel-L2 vs FP64 | rotation bin | FP64 argmax in the bin's slice |")
    for prec, (err, b, same) in rows.items():
        print(f"| {NAMES[prec]} | {err:.3e} | {b} | {'same' if same else 'differs'} |")
    for prec, (err, b, same) in rows.items():
        assert err <= REL_L2, NAMES[prec]
        assert b == rows[0][1], NAMES[prec]
        assert same, NAMES[prec]
    c32.close()
