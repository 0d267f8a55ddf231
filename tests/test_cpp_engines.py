"""The C++ engine classes (dspsr-kanyixia_b200/cpp/) that mirror DSPSR's CUDA
engines compile against the C ABI, and drive the GPU correctly."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "dspsr-kanyixia_b200")
OUT = os.path.join(ROOT, "tests", "cpp", "_build")
EXE = os.path.join(OUT, "engines_main")


def build():
    os.makedirs(OUT, exist_ok=True)
    cmd = ["/usr/local/cuda/bin/nvcc", "-std=c++17", "-O2", "-x", "cu",
           "-gencode", "arch=compute_100a,code=sm_100a",
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(PKG, "cpp"),
           os.path.join(PKG, "cpp", "dsp_b200_engines.cpp"),
           os.path.join(ROOT, "tests", "cpp", "engines_main.cpp"),
           "-L", os.path.join(PKG, "lib"), "-ldspsr_b200",
           "-Xlinker", "-rpath=" + os.path.join(PKG, "lib"), "-o", EXE]
    subprocess.run(cmd, check=True, capture_output=True, text=True)


def test_cpp_engines_build(b2):
    build()
    assert os.path.exists(EXE)


@pytest.mark.gpu
def test_cpp_engines_run(b2):
    if not os.path.exists(EXE):
        build()
    r = subprocess.run([EXE], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "ALL OK" in r.stdout, r.stdout + r.stderr
