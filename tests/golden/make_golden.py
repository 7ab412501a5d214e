"""Generates the golden fixtures in tests/golden/ by running the reference's
own SOFT sources (oracle/_ref, built by oracle/Makefile from the reference
tree) on seeded inputs.  Run once where the reference tree exists:

    python tests/golden/make_golden.py

The fixtures then pin the oracle (and through it the CUDA path) on machines
without the reference tree.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def main():
    O.build(ref=True)
    rng = np.random.default_rng(20240)
    out = {}
    # SOFT forward SHT (FST_semi_memo) of a seeded real signal, B = 8
    bw = 8
    sig = rng.standard_normal(4 * bw * bw)
    out["sht_b8_signal"] = sig
    out["sht_b8_coef"] = O.ref_sht(sig, bw)
    # Laplace spherical correlation (4 channels, last all zero), B = 8
    f = rng.standard_normal((4, 4 * bw * bw))
    g = rng.standard_normal((4, 4 * bw * bw))
    f[3] = 0.0
    g[3] = 0.0
    corr, vol = O.ref_spherical_correlation(f, g, bw, volume=True)
    out["sph_b8_f"] = f
    out["sph_b8_g"] = g
    out["sph_b8_corr"] = corr
    out["sph_b8_argmax"] = np.int64(np.argmax(corr))
    # single-channel SphericalCorrelation, B = 6, bw_out = 8 (zero padding 2)
    f1 = rng.standard_normal((1, 4 * 36))
    g1 = rng.standard_normal((1, 4 * 36))
    c1 = O.ref_spherical_correlation(f1, g1, 6, 8)
    out["sph1_b6p2_f"] = f1
    out["sph1_b6p2_g"] = g1
    out["sph1_b6p2_corr"] = c1
    # Laplace spatial correlation N = 6, 4 channels
    N = 6
    fs = rng.standard_normal((4, N ** 3))
    gs = rng.standard_normal((4, N ** 3))
    out["spat_n6_f"] = fs
    out["spat_n6_g"] = gs
    out["spat_n6_c"] = O.ref_spatial_correlation(fs, gs, N, laplace=True)
    np.savez_compressed(os.path.join(OUT, "soft_reference_small.npz"), **out)
    print("wrote", os.path.join(OUT, "soft_reference_small.npz"))


if __name__ == "__main__":
    main()
