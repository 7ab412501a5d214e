"""The C++ ingest drop-in PlyHelper (include/phaser_gpu.hpp) compiles against
the C ABI and reads an Ouster-style PLY on the host (no GPU needed)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "ply_test.cc")
LIBDIR = os.path.join(ROOT, "phaser_b200", "_lib")


def test_cpp_ply_helper(tmp_path):
    from phaser_b200 import build
    build.build()
    exe = str(tmp_path / "ply_test")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I" + os.path.join(ROOT, "include"), SRC,
           "-L" + LIBDIR, "-lphaser_gpu", "-Wl,-rpath," + LIBDIR, "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    r = subprocess.run([exe, str(tmp_path / "scan.ply")], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ply_fields 6" in r.stdout and "ply_missing_rejected" in r.stdout
    assert r.stdout.strip().endswith("ok")
