"""The three shared-memory FFT engines against numpy, rows and columns,
forward and inverse (tolerance: FP32 transform error), through a test-only
library (tests/cuda/fft_selftest.cu) linked against the product library."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
_LIB = None


def _selftest_lib():
    """Builds (when stale) and loads tests/_build/libphaser_fft_selftest.so."""
    global _LIB
    if _LIB is not None:
        return _LIB
    from phaser_b200 import build
    prod = build.build()
    src = os.path.join(HERE, "cuda", "fft_selftest.cu")
    out_dir = os.path.join(HERE, "_build")
    os.makedirs(out_dir, exist_ok=True)
    so = os.path.join(out_dir, "libphaser_fft_selftest.so")
    deps = [src, prod] + [os.path.join(build.CSRC, f) for f in os.listdir(build.CSRC) if f.endswith((".cuh", ".h"))]
    if not os.path.exists(so) or any(os.path.getmtime(d) > os.path.getmtime(so) for d in deps):
        libdir = os.path.dirname(prod)
        subprocess.run([build.nvcc()] + build.ARCH + build.NVCC_FLAGS +
                       ["-shared", src, "-o", so, "-L" + libdir, "-lphaser_gpu", "-Xlinker", "-rpath=" + libdir],
                       check=True, capture_output=True, text=True)
    lib = C.CDLL(so)
    lib.phgpu_selftest_fft.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]
    _LIB = lib
    return lib


class _Native:
    @staticmethod
    def selftest_fft(x, inverse=False, columns=False, engine=2):
        a = np.ascontiguousarray(x, np.complex64).copy()  # transformed in place
        ntrans, n = a.shape
        rc = _selftest_lib().phgpu_selftest_fft(n, ntrans, 1 if inverse else 0, 1 if columns else 0, engine,
                                                a.ctypes.data)
        if rc != 0:
            raise RuntimeError(f"phgpu_selftest_fft failed ({rc})")
        return a

SIZES = [32, 64, 100, 128, 200, 256, 512]


@pytest.mark.parametrize("engine", [0, 1, 2])
@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("columns", [False, True])
@pytest.mark.parametrize("inverse", [False, True])
def test_fft_engine(engine, n, columns, inverse):
    native = _Native
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
    native = _Native
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
    native = _Native
    rng = np.random.default_rng(320)
    x = (rng.standard_normal((24, 320)) + 1j * rng.standard_normal((24, 320))).astype(np.complex64)
    y = native.selftest_fft(x, inverse=inverse, columns=columns, engine=1)
    ref = np.fft.ifft(x.astype(np.complex128), axis=1) * 320 if inverse else np.fft.fft(x.astype(np.complex128), axis=1)
    assert np.abs(y - ref).max() / np.abs(ref).max() < 5e-6
