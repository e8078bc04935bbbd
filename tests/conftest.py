"""pytest configuration: the `gpu` marker and shared helpers.

CPU tests (`-m "not gpu"`) cover the oracle against the reference's pinned
numbers, the host logic of libllg.so (geometry builders, knob parser, ABI
surface) and multi-process host paths.  `-m gpu` tests call the CUDA path
through the C ABI and compare it with the oracle.
"""
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "gpu-micromagnetics-irregular_b200")
for p in (PKG, os.path.join(REPO, "oracle"), os.path.join(REPO, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the libllg.so kernels")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle_lib():
    import binding
    binding.build()
    return binding


@pytest.fixture(scope="session")
def llg_lib():
    import llg
    if not os.path.exists(llg.LIB_PATH):
        import subprocess
        subprocess.run(["make", "-s", "-C", PKG], check=True)
    return llg


@pytest.fixture(scope="session")
def gpu():
    if not has_gpu():
        pytest.fail("GPU test selected but no CUDA device is visible")
    import torch
    return torch.device("cuda:0")


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    scale = max(float(np.abs(b).max()), 1e-300)
    return float(np.abs(a - b).max() / scale)
