"""The two-for-one transform identities the kernels rely on, restated with
numpy FFTs (FP64) on random data.

* SO(3) gamma transform (k_so3_c2r_tail in phaser_b200/csrc/k_so3.cu): a row
  holds X[b] = conj(u_b), X[n - b] = u_b for 0 < b < n/2, X[0] = conj(u_0)
  and X[n/2] = 0, and only the real part of its inverse DFT is used.  Two
  rows a, b go through one complex inverse DFT of Z = X_a' + i X_b', where X'
  is X with its DC term made real: Re of each row's inverse equals the real
  and imaginary parts of Z's inverse.
* SHT phi transform (k_sht_phi in phaser_b200/csrc/k_sht.cu): two real rows
  x_a, x_b through one forward DFT of z = x_a + i x_b, split as
  X_a[m] = (Z[m] + conj Z[-m]) / 2, X_b[m] = (Z[m] - conj Z[-m]) / 2i.
"""
import numpy as np
import pytest


def row_spectrum(u, n):
    X = np.zeros(n, complex)
    X[0] = np.conj(u[0])
    for b in range(1, n // 2):
        X[b] = np.conj(u[b])
        X[n - b] = u[b]
    return X


@pytest.mark.parametrize("n", [8, 64, 200, 320])
def test_gamma_rows_two_per_transform(n):
    rng = np.random.default_rng(n)
    half = n // 2
    ua = rng.standard_normal(half) + 1j * rng.standard_normal(half)
    ub = rng.standard_normal(half) + 1j * rng.standard_normal(half)
    # what the one-row-per-transform kernel computes: Re of the inverse DFT
    # (numpy's ifft carries 1/n; both sides use it)
    ra = np.fft.ifft(row_spectrum(ua, n)).real
    rb = np.fft.ifft(row_spectrum(ub, n)).real
    # the packed row as k_so3_c2r_tail fills it
    Z = np.zeros(n, complex)
    Z[0] = ua[0].real + 1j * ub[0].real
    for b in range(1, half):
        Z[b] = (ua[b].real + ub[b].imag) + 1j * (ub[b].real - ua[b].imag)  # conj(ua) + i conj(ub)
        Z[n - b] = (ua[b].real - ub[b].imag) + 1j * (ua[b].imag + ub[b].real)  # ua + i ub
    z = np.fft.ifft(Z)
    assert np.allclose(z.real, ra, atol=1e-13)
    assert np.allclose(z.imag, rb, atol=1e-13)


@pytest.mark.parametrize("n", [4, 50, 200, 256])
def test_phi_rows_two_per_transform(n):
    rng = np.random.default_rng(n + 1)
    xa, xb = rng.standard_normal(n), rng.standard_normal(n)
    Z = np.fft.fft(xa + 1j * xb)
    m = np.arange(n // 2)
    zb = Z[(-m) % n]
    Xa = 0.5 * ((Z[m].real + zb.real) + 1j * (Z[m].imag - zb.imag))
    Xb = 0.5 * ((Z[m].imag + zb.imag) + 1j * (zb.real - Z[m].real))
    assert np.allclose(Xa, np.fft.fft(xa)[m], atol=1e-12)
    assert np.allclose(Xb, np.fft.fft(xb)[m], atol=1e-12)
