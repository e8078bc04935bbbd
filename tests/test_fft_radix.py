"""The in-register DFT butterflies of the FFT core, checked on the CPU.

tests/native/fft_radix_check.cu includes csrc/dev_fft.cuh (whose butterflies
are __host__ __device__), runs every fixed radix (2, 3, 4, 5, 6, 8, 12, 16) in
both directions in FP64 and FP32 on the host and compares each with a direct
DFT in long double: rel 1e-15 (FP64) and 1e-6 (FP32).  The Stockham passes
that use them are checked on the GPU by the demag parity tests.
"""
import os
import shutil
import subprocess

import pytest

from conftest import PKG, REPO


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="nvcc not available")
def test_fixed_radix_butterflies(tmp_path):
    exe = tmp_path / "fft_radix_check"
    src = os.path.join(REPO, "tests", "native", "fft_radix_check.cu")
    subprocess.run(["nvcc", "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-Wno-deprecated-gpu-targets", "-I" + os.path.join(PKG, "csrc"), src, "-o", str(exe)],
                   check=True, capture_output=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    print(out.stdout)
    assert out.returncode == 0, out.stdout
    assert out.stdout.count("rel err") == 32
