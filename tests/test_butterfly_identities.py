"""The small-DFT butterflies of the FFT engine and the shared-memory layout of
the translation z pass, restated in numpy on the host.

* phaser_b200/csrc/fft.cuh, dft_small<R, INV>: the radix-2/3/4/5/8
  butterflies written as packed-pair sums (both components of a complex sum,
  or of a complex times a real constant, in one FADD2 / FFMA2 / FMUL2) and
  per-component rotations by +-i (rot_pm).  Restated step by step in FP64
  they must equal the DFT sum_j x_j exp(sg 2 pi i j k / R), sg = -1 forward
  and +1 inverse.
* phaser_b200/csrc/k_spatial.cu, k_fuse_z: a tile row holds A slots of Wt
  complex (A * Wt * 8 bytes, a multiple of 128 at Wt = 8), so every row
  starts on bank 0.  Odd rows keep their product in slot 1 (row-parity
  slots) and load their two sides in the opposite order; the model below
  counts shared-memory wavefronts (32 banks of 4 bytes, a 64-bit access
  served per half-warp) for the fusion loads and the inverse transform's
  loads, with and without the slots.
"""
import numpy as np
import pytest


def rot_pm(a, d, inv):
    """a + i sg d and a - i sg d (fft.cuh rot_pm)."""
    if inv:
        return complex(a.real - d.imag, a.imag + d.real), complex(a.real + d.imag, a.imag - d.real)
    return complex(a.real + d.imag, a.imag - d.real), complex(a.real - d.imag, a.imag + d.real)


def dft_small(x, inv):
    """dft_small<R, INV> of fft.cuh, operation by operation."""
    x = list(x)
    R = len(x)
    sg = 1.0 if inv else -1.0
    if R == 2:
        return [x[0] + x[1], x[0] - x[1]]
    if R == 3:
        s3 = 0.86602540378443864676
        t1, t2 = x[1] + x[2], x[1] - x[2]
        y0 = x[0] + t1
        m1 = x[0] + (-0.5) * t1
        p, m = rot_pm(m1, s3 * t2, inv)
        return [y0, p, m]
    if R == 4:
        t0, t1, t2, d = x[0] + x[2], x[0] - x[2], x[1] + x[3], x[1] - x[3]
        p, m = rot_pm(t1, d, inv)
        return [t0 + t2, p, t0 - t2, m]
    if R == 5:
        c1, c2 = 0.30901699437494742410, -0.80901699437494742410
        s1, s2 = 0.95105651629515357212, 0.58778525229247312917
        t1, t2, t3, t4 = x[1] + x[4], x[2] + x[3], x[1] - x[4], x[2] - x[3]
        y0 = x[0] + (t1 + t2)
        a1 = x[0] + c1 * t1 + c2 * t2
        a2 = x[0] + c2 * t1 + c1 * t2
        b1 = s1 * t3 + s2 * t4
        b2 = s2 * t3 - s1 * t4
        y1, y4 = rot_pm(a1, b1, inv)
        y2, y3 = rot_pm(a2, b2, inv)
        return [y0, y1, y2, y3, y4]
    if R == 8:
        e = dft_small([x[0], x[2], x[4], x[6]], inv)
        o = dft_small([x[1], x[3], x[5], x[7]], inv)
        h = 0.70710678118654752440
        o1 = h * complex(o[1].real - sg * o[1].imag, o[1].imag + sg * o[1].real)
        p3 = complex(o[3].real + sg * o[3].imag, sg * o[3].real - o[3].imag)
        o3 = complex(-h * p3.real, h * p3.imag)
        x2, x6 = rot_pm(e[2], o[2], inv)
        return [e[0] + o[0], e[1] + o1, x2, e[3] + o3, e[0] - o[0], e[1] - o1, x6, e[3] - o3]
    raise ValueError(R)


@pytest.mark.parametrize("R", [2, 3, 4, 5, 8])
@pytest.mark.parametrize("inv", [False, True])
def test_small_dft_equals_the_dft(R, inv):
    rng = np.random.default_rng(R + 10 * inv)
    for _ in range(20):
        x = rng.standard_normal(R) + 1j * rng.standard_normal(R)
        want = np.fft.ifft(x) * R if inv else np.fft.fft(x)
        got = np.array(dft_small(x, inv))
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-12 * max(1.0, np.abs(x).sum()))


def _wavefronts(addrs):
    """Shared-memory wavefronts of one warp's 64-bit access (addresses in
    float2 units, None = inactive lane): per half-warp, the most distinct
    words any one bank must serve."""
    total = 0
    for h in range(2):
        banks = {}
        for a in addrs[16 * h:16 * h + 16]:
            if a is None:
                continue
            for w in (2 * a, 2 * a + 1):
                banks.setdefault(w % 32, set()).add(w)
        total += max((len(v) for v in banks.values()), default=0)
    return total


N, C, WT, THREADS = 200, 3, 8, 512
A = 2 * C
ROWLEN = A * WT


def _fusion_wavefronts(podd):
    """Mean wavefronts per load instruction of the fusion pass: element
    e -> (row e / Wt, column e % Wt); each channel c loads side f (slot c)
    and side g (slot C + c), odd rows the other way round when podd."""
    per = []
    for w0 in range(0, N * WT, 32):
        for c in range(C):
            for first in (True, False):
                addrs = []
                for e in range(w0, w0 + 32):
                    zp, t = divmod(e, WT)
                    odd = bool(podd) and zp % 2 == 1
                    slot = (C + c if odd else c) if first else (c if odd else C + c)
                    addrs.append(zp * ROWLEN + slot * WT + t)
                per.append(_wavefronts(addrs))
    return np.mean(per)


def _inverse_wavefronts(podd):
    """Mean wavefronts per load of the inverse z transform over the Wt
    product columns (column-resident mapping: thread -> column tid % Wt,
    butterfly group tid / Wt), element i of a column at
    i * rowlen + (i odd ? podd : 0) + t."""
    stages = [(5, 5), (5, 25), (8, 200)]  # inverse order of 200 = 8 * 5 * 5
    groups = THREADS // WT
    per = []
    for R, L in stages:
        m, nb = L // R, N // R
        for w in range(THREADS // 32):
            for k in range(-(-nb // groups)):
                for j in range(R):
                    addrs = []
                    for lane in range(32):
                        tid = 32 * w + lane
                        t, g = tid % WT, tid // WT
                        bf = g + k * groups
                        if bf >= nb:
                            addrs.append(None)
                            continue
                        blk, j2 = divmod(bf, m)
                        r = blk * L + j2 + j * m
                        addrs.append(t + r * ROWLEN + (r % 2) * podd)
                    if any(a is not None for a in addrs):
                        per.append(_wavefronts(addrs))
    return np.mean(per)


def test_row_parity_slots_remove_the_bank_conflicts():
    assert (ROWLEN * 8) % 128 == 0  # every row starts on bank 0
    assert _fusion_wavefronts(0) == pytest.approx(4.0)
    assert _fusion_wavefronts(WT) == pytest.approx(2.0)  # the minimum for 32 x 8 bytes
    assert _inverse_wavefronts(0) > 3.5
    assert _inverse_wavefronts(WT) < 2.0 + 1e-9


def test_row_parity_slots_are_a_layout_of_the_product_column():
    """Every (row, column) of the product lands in its own word of the tile,
    inside its row, in slot 0 (even rows) or slot 1 (odd rows)."""
    seen = set()
    for i in range(N):
        for t in range(WT):
            a = i * ROWLEN + (i % 2) * WT + t
            assert i * ROWLEN <= a < (i + 1) * ROWLEN
            assert (a - i * ROWLEN) // WT == i % 2
            seen.add(a)
    assert len(seen) == N * WT
