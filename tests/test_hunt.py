"""The blackbody point-wise path hunts phase_o from each thread's previous
bracket (hunt_from, csrc/device.cuh) and the phase-major walk steps to it
(walk_bracket); on a non-decreasing phase_o both must give the same clamped
index and fraction as vhunt's bisection, from any start.
Checked on the host: tests/hunt_check.cu compiles the same device header with
nvcc and compares both on random arrays with repeated values."""
import os
import subprocess

import pytest

from gpu_ppm_b200 import build as B

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def test_hunt_from_matches_bisection(tmp_path):
    if not os.path.exists(B.NVCC):
        pytest.skip("nvcc not available")
    exe = tmp_path / "hunt_check"
    subprocess.run([B.NVCC, "-std=c++17", "-O2", *B.ARCH, "-I", os.path.join(ROOT, "include"), "-I", B.CSRC,
                    os.path.join(HERE, "hunt_check.cu"), "-o", str(exe)], check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    cases, bad = int(out[0]), int(out[1])
    assert cases == 320000 and bad == 0
