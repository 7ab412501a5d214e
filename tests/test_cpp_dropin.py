"""The header-only C++ drop-ins (include/phaser_gpu.hpp) compile against the
C ABI and, on a GPU, reproduce the reference's spatial known answer."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "dropin_test.cc")
LIBDIR = os.path.join(ROOT, "phaser_b200", "_lib")


def _build(tmp_path):
    from phaser_b200 import build
    build.build()
    exe = str(tmp_path / "dropin_test")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I" + os.path.join(ROOT, "include"), SRC,
           "-L" + LIBDIR, "-lphaser_gpu", "-Wl,-rpath," + LIBDIR, "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_cpp_dropin_compiles_and_links(tmp_path):
    exe = _build(tmp_path)
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_cpp_dropin_runs(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "spatial_delta 0 2 0" in r.stdout
    assert r.stdout.strip().endswith("ok")
