"""The bound behind the exact 1-NN row sweep (phaser_b200/csrc/k_sample.cu),
checked by brute force on the CPU.

The sweep keeps hb >= sin^2(beta / 2) for the angle beta of the best squared
chord (inflated by 1e-4 rad), visits a row while hav of its colatitude
distance stays within hb, and scans the columns within the haversine-law
window k of the row.  The search is exact only if every point whose float
squared chord to the direction does not exceed the best one lies in a visited
row and inside that row's window.  This test restates the bound's arithmetic
(float32, the kernel's tables and margins) and checks that claim for random
directions of the Driscoll-Healy grid against points scattered around them at
scales from 1e-4 rad to the whole sphere, binned the way the projection bins
them.
"""
import numpy as np
import pytest

MARGIN = np.float32(1e-4)


def tables(n2b):
    w = np.pi / n2b
    r = np.arange(n2b + 1)
    sin_tab = np.maximum(np.sin(r * w).astype(np.float32) - np.float32(1e-5), np.float32(0))
    sin_tab[n2b] = 0
    d = np.arange(n2b + 1)
    hav = (np.sin(0.5 * (d - 0.5) * w) ** 2).astype(np.float32) * np.float32(1 - 1e-4)
    hav[0] = 0
    return sin_tab, hav


def hav_of_l2(best):
    best = np.float32(best)
    if not best < np.float32(3.99):
        return np.float32(2)
    s = np.float32(0.5) * np.sqrt(best) * (np.float32(1) + MARGIN) + np.float32(0.5) * MARGIN
    return np.float32(2) if s >= 1 else np.float32(s * s)


def row_window(r, d, n2b, w, stq, hb, sin_tab, hav_tab):
    if hb >= 1:
        return n2b
    num = np.float32(hb - hav_tab[d])
    den = np.float32(min(sin_tab[r], sin_tab[r + 1]) * stq)
    if not num < den:
        return n2b
    if num <= 0:
        return 0
    e = np.float32(2) * np.arcsin(np.sqrt(np.float32(num / den))) + MARGIN
    kf = np.float32(e / (np.float32(2) * w) + np.float32(0.5))
    return n2b if kf >= n2b else int(kf)


def grid_direction(i, j, bw):
    th = np.float32(np.pi * (2 * i + 1) / (4 * bw))
    ph = np.float32(2 * np.pi * j / (2 * bw))
    return np.array([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], dtype=np.float32)


def project_and_bin(v, n2b):
    """Unit direction and (row, column) bin of each point, as k_project."""
    v = v.astype(np.float32)
    dist = np.sqrt((v.astype(np.float64) ** 2).sum(axis=1))
    oz = (v[:, 2] / dist).astype(np.float32)
    tx = np.arccos(oz.astype(np.float64)).astype(np.float32).astype(np.float64)
    ty = np.mod(np.arctan2(v[:, 1].astype(np.float64), v[:, 0].astype(np.float64)).astype(np.float32)
                + 2 * np.pi, 2 * np.pi)
    proj = np.stack([np.sin(tx) * np.cos(ty), np.sin(tx) * np.sin(ty), np.cos(tx)], axis=1).astype(np.float32)
    w = np.pi / n2b
    bi = np.clip((tx / w).astype(np.int64), 0, n2b - 1)
    bj = np.floor(ty / (2 * w) + 0.5).astype(np.int64)
    bj = np.where(bj >= n2b, bj - n2b, np.maximum(bj, 0))
    return proj, bi, bj


def dist2(q, p):
    d = (q[None, :] - p).astype(np.float32)
    return ((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]).astype(np.float32) + d[:, 2] * d[:, 2]).astype(np.float32)


@pytest.mark.parametrize("bw", [4, 16, 50, 100])
def test_window_covers_every_point_within_the_bound(bw):
    rng = np.random.default_rng(bw)
    n2b = 2 * bw
    w = np.float32(np.float32(3.14159265358979) / np.float32(n2b))
    sin_tab, hav_tab = tables(n2b)
    checked = 0
    for _ in range(60):
        i, j = int(rng.integers(n2b)), int(rng.integers(n2b))
        q = grid_direction(i, j, bw)
        stq = np.float32(max(np.float32(np.sin(np.float32((i + 0.5) * w))) - np.float32(1e-5), 0))
        for scale in (1e-4, 1e-3, 1e-2, 0.1, 0.5, 3.0):
            pts = q[None, :].astype(np.float64) + rng.standard_normal((400, 3)) * scale
            proj, bi, bj = project_and_bin(pts, n2b)
            d2 = dist2(q, proj)
            # bounds: the chords of some of the points themselves (ties
            # included) and a few values in between
            for best in np.concatenate([rng.choice(d2, 6), np.float32([np.median(d2) * 0.5])]):
                hb = hav_of_l2(best)
                inside = d2 <= best
                for r, c in zip(bi[inside], bj[inside]):
                    d = abs(int(r) - i)
                    assert hav_tab[d] <= hb, (bw, i, j, r, best)
                    k = row_window(int(r), d, n2b, w, stq, hb, sin_tab, hav_tab)
                    dc = abs(int(c) - j)
                    dc = min(dc, n2b - dc)
                    assert 2 * k + 1 >= n2b or dc <= k, (bw, i, j, r, c, k, best)
                    checked += 1
    assert checked > 1000
