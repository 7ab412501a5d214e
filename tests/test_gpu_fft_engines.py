"""The three shared-memory FFT engines against numpy, rows and columns,
forward and inverse (tolerance: FP32 transform error)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIZES = [32, 64, 100, 128, 200, 256, 512]


@pytest.mark.parametrize("engine", [0, 1, 2])
@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("columns", [False, True])
@pytest.mark.parametrize("inverse", [False, True])
def test_fft_engine(engine, n, columns, inverse):
    from phaser_b200 import native
    rng = np.random.default_rng(n + 7 * engine)
    ntrans = max(1, min(24, (200 * 1024) // ((n + 1) * 8)))
    x = (rng.standard_normal((ntrans, n)) + 1j * rng.standard_normal((ntrans, n))).astype(np.complex64)
    y = native.selftest_fft(x, inverse=inverse, columns=columns, engine=engine)
    ref = np.fft.ifft(x.astype(np.complex128), axis=1) * n if inverse else np.fft.fft(x.astype(np.complex128), axis=1)
    err = np.abs(y - ref).max() / np.abs(ref).max()
    assert err < 5e-6, err


@pytest.mark.parametrize("n", [3, 12, 38, 127, 134, 201, 254])
@pytest.mark.parametrize("columns", [False, True])
def test_fft_runtime_engine_odd_lengths(n, columns):
    # large prime factors (19, 67, 127) run through the generic radix stage
    from phaser_b200 import native
    rng = np.random.default_rng(n)
    x = (rng.standard_normal((7, n)) + 1j * rng.standard_normal((7, n))).astype(np.complex64)
    for inverse in (False, True):
        y = native.selftest_fft(x, inverse=inverse, columns=columns, engine=0)
        ref = np.fft.ifft(x.astype(np.complex128), axis=1) * n if inverse else np.fft.fft(x.astype(np.complex128), axis=1)
        assert np.abs(y - ref).max() / np.abs(ref).max() < 5e-6


@pytest.mark.parametrize("columns", [False, True])
@pytest.mark.parametrize("inverse", [False, True])
def test_fft_compile_time_plan_320(columns, inverse):
    # 2 bw_out of the reference run script's rotation (B = 150, padding 10)
    from phaser_b200 import native
    rng = np.random.default_rng(320)
    x = (rng.standard_normal((24, 320)) + 1j * rng.standard_normal((24, 320))).astype(np.complex64)
    y = native.selftest_fft(x, inverse=inverse, columns=columns, engine=1)
    ref = np.fft.ifft(x.astype(np.complex128), axis=1) * 320 if inverse else np.fft.fft(x.astype(np.complex128), axis=1)
    assert np.abs(y - ref).max() / np.abs(ref).max() < 5e-6
