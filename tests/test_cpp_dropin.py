"""The header-only C++ drop-in (include/roger_b200/ocl_dropin.hpp) compiles against the C ABI
(CPU) and round-trips an image exactly through OCLEncoder<short> / OCLDecoder<short> (GPU)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "roger_b200")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def _build(tmp_path):
    from roger_b200 import _lib
    _lib.lib()  # builds libj2kb200.so if needed
    exe = str(tmp_path / "dropin_roundtrip")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-I", os.path.join(ROOT, "include"), "-I",
           os.path.join(CUDA, "include"), os.path.join(ROOT, "tests", "cpp", "dropin_roundtrip.cpp"),
           "-o", exe, "-L", LIBDIR, "-lj2kb200", "-Wl,-rpath," + LIBDIR, "-L", os.path.join(CUDA, "lib64"),
           "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


@pytest.mark.skipif(shutil.which("g++") is None, reason="no g++")
def test_dropin_header_compiles_and_links(tmp_path):
    assert os.path.exists(_build(tmp_path))


@pytest.mark.gpu
def test_dropin_round_trip_on_gpu(tmp_path):
    exe = _build(tmp_path)
    for w, h in [(301, 197), (64, 64), (1024, 33)]:
        r = subprocess.run([exe, str(w), str(h)], capture_output=True, text=True, timeout=120)
        assert r.returncode == 0, r.stdout + r.stderr
        assert r.stdout.startswith("ok")
