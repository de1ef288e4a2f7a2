"""Test configuration: the `gpu` marker and the in-tree builds.

GPU tests call the CUDA path through the C ABI (libfd2.so).  CPU tests
cover the oracle against the reference's own C functions and golden
fixtures, the host logic, and the library's exported symbols.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def _ensure_built():
    lib = os.path.join(ROOT, "hybridmantis_b200", "lib", "libfd2.so")
    orc = os.path.join(ROOT, "oracle", "_build", "libfd2oracle.so")
    if not os.path.exists(orc):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "all"], check=True)
    if not os.path.exists(lib):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "hybridmantis_b200"), "-j8"], check=True)


_ensure_built()


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def require_gpu():
    if not gpu_available():
        pytest.fail("GPU test selected but no CUDA device is visible")
