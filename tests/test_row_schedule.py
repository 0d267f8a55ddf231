"""The FP32 convolution row kernel's pass schedule (Row32 in
csrc/fft_core.cuh), run on the CPU one thread and one barrier phase at a
time: forward 4096- and 8192-point transforms and the convolution row
(forward, x H, inverse) against an FP64 DFT, and every shared-memory access
of a half-warp free of bank conflicts."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "dspsr-kanyixia_b200", "csrc")
OUT = os.path.join(ROOT, "tests", "cpp", "_build")
EXE = os.path.join(OUT, "row32_main")


def test_row32_schedule():
    os.makedirs(OUT, exist_ok=True)
    subprocess.run(["g++", "-O2", "-std=c++17", "-I/usr/local/cuda/include", "-I", CSRC,
                    os.path.join(ROOT, "tests", "cpp", "row32_main.cpp"), "-o", EXE],
                   check=True, capture_output=True, text=True)
    r = subprocess.run([EXE], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = [l for l in r.stdout.splitlines() if l.startswith("row32")]
    assert len(lines) == 2
    for l in lines:
        f = dict(kv.split("=") for kv in l.split()[1:])
        assert float(f["forward_rel_rms"]) < 1e-6
        assert float(f["conv_rel_rms"]) < 1e-6
        assert int(f["bank_conflicts"]) == 0
