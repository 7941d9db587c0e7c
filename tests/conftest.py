"""Shared test setup: import paths, the `gpu` marker, and build helpers.

`-m "not gpu"` tests run on any machine (oracle vs golden vectors, the C ABI
library loading and exporting its symbols); `-m gpu` tests call the CUDA
kernels through the C ABI and compare with the oracle.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "hpl-ai_b200")
for p in (PKG, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (sm_100a, B200)")


def build_library():
    """Build libhplai.so in-tree if it is missing (nvcc cross-compiles)."""
    lib = os.path.join(PKG, "libhplai.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-s", "-C", PKG, "-j4"], check=True)
    return lib


@pytest.fixture(scope="session")
def hplai():
    build_library()
    import hplai as mod
    return mod


@pytest.fixture(scope="session")
def oracle():
    import oracle as mod
    return mod


@pytest.fixture(scope="session")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("GPU test collected but CUDA is not available")
    return torch
